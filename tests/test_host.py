"""Host-side logic of the drop-in, checked on the CPU.

The product builds its filter constants in FP64 on the host; these tests
check them against the golden windows and, through a NumPy model of the
device filter (the same power-of-two embedding and two-rows-per-transform
packing the kernel uses), against the oracle's filter.
"""
import numpy as np
import pytest

from algotom_b200 import _native as nat
from algotom_b200 import phantom
from algotom_b200.rec import windows as W
from oracle import fbp_oracle as O

WINDOWS = ["hann", "bartlett", "blackman", "hamming", "nuttall", "parzen",
           "triang", None]


def test_product_windows_match_reference(golden):
    g = golden("windows")
    for w in (64, 65):
        for name in WINDOWS:
            np.testing.assert_array_equal(W.make_smoothing_window(name, w),
                                          g["smooth__%s__%d" % (name, w)])
            np.testing.assert_allclose(W.make_2d_ramp_window(2, w, name),
                                       g["ramp2d__%s__%d" % (name, w)],
                                       rtol=0, atol=1e-15)
        for name in ("hann", None):
            np.testing.assert_allclose(W.make_circular_ramp_window(w, name),
                                       g["circ__%s__%d" % (name, w)],
                                       rtol=0, atol=1e-14)
    for w, ratio in ((65, 1.0), (64, 0.7), (97, 0.93)):
        np.testing.assert_array_equal(W.make_circle_mask(w, ratio),
                                      g["mask__%d__%s" % (w, ratio)])


def _device_filter_model(x2, pad, mode, window_row, m=None):
    """NumPy model of atb_filter_rows for two rows (transform length m:
    atb_filter_length's choice by default)."""
    ncol = x2.shape[1]
    if m is None:
        m = nat.call("atb_filter_length", ncol, pad)
    spec = W.row_filter_spectrum(window_row, ncol, pad, m)[0]
    xp = np.pad(x2, ((0, 0), (pad, pad)), mode=mode)
    z = np.zeros(m, complex)
    z[:ncol + 2 * pad] = xp[0] + 1j * xp[1]
    w = np.fft.fft(np.conj(np.fft.fft(z) * spec))
    return np.stack([w.real[pad:pad + ncol], -w.imag[pad:pad + ncol]])


@pytest.mark.parametrize("ncol,pad", [(96, 14), (81, 12), (50, 0), (33, 80)])
@pytest.mark.parametrize("name", ["hann", None, "parzen"])
def test_spectrum_embedding_reproduces_filter(ncol, pad, name):
    """Every exact length: N itself, the smallest embedding and a longer
    one, against the oracle's length-N filter."""
    rng = np.random.default_rng(ncol + pad)
    x = rng.standard_normal((2, ncol))
    n = ncol + 2 * pad
    ref = O.apply_ramp_filter(x, None, name, pad, "edge")
    for m in (None, n, n + ncol - 1, 2 * (n + ncol)):
        got = _device_filter_model(x, pad, "edge",
                                   W.ramp_window_row(n, name), m)
        assert O.rel_l2(got, ref) < 1e-6   # complex64 spectrum


def test_spectrum_rejects_short_fft():
    with pytest.raises(ValueError):
        W.row_filter_spectrum(W.ramp_window_row(100, "hann"), 80, 10, 128)
    with pytest.raises(ValueError):
        W.row_filter_spectrum(W.ramp_window_row(100, "hann"), 80, 10, 101)


def test_filter_twiddles():
    """atb_filter_twiddles: each stage's exp(-2 pi i r k / (Ns R)) at
    Ns - 1 + k (R - 1) + r - 1, the stages in the kernel's radix order."""
    def radices(n):
        out, m = [], n
        while m % 16 == 0:
            out.append(16)
            m //= 16
        for q in (8, 4, 2):
            if m % q == 0:
                out.append(q)
                m //= q
        for q in (13, 11, 7, 5, 3):
            while m % q == 0:
                out.append(q)
                m //= q
        return out
    for n in (64, 60, 2860, 2560, 4410):
        t = np.empty(2 * n, np.float32)
        nat.call("atb_filter_twiddles", n, t.ctypes.data)
        t = t.view(np.complex64)
        ref = np.zeros(n, np.complex128)
        ns = 1
        for r_ in radices(n):
            for k in range(ns):
                for r in range(1, r_):
                    ref[ns - 1 + k * (r_ - 1) + r - 1] = np.exp(
                        -2j * np.pi * r * k / (ns * r_))
            ns *= r_
        ref[n - 1] = 1.0
        np.testing.assert_allclose(t, ref, atol=1e-7)
    lib = nat.load()
    t = np.empty(2 * 17, np.float32)
    assert lib.atb_filter_twiddles(17, t.ctypes.data) == -1  # no plan for 17
    assert lib.atb_filter_twiddles(16, None) == -1


def test_phantom_sinogram_is_exact_line_integral():
    """Exact invariants of the analytic projections of one ellipse: every
    angle carries the same mass mu/n * pi A B, centred on the projected
    ellipse centre."""
    x0, y0, a, b, phi, mu = 5.0, -3.0, 20.0, 9.0, 0.4, 0.7
    params = np.array([[x0, y0, a, b, phi, mu]])
    n = 96
    ang = np.linspace(0.0, np.pi, 7)
    sino = phantom.analytic_sinogram(params, ang, n, 47.5, size=n)
    j = np.arange(n)
    for i, th in enumerate(ang):
        mass = sino[i].sum()
        assert mass == pytest.approx(mu / n * np.pi * a * b, rel=1e-2)
        cen = (sino[i] * j).sum() / mass
        assert cen == pytest.approx(x0 * np.cos(th) - y0 * np.sin(th) + 47.5,
                                    abs=0.1)
    # and the FBP of it reproduces the rasterised ellipse
    rec = O.fbp_reconstruction(phantom.analytic_sinogram(
        params, np.linspace(0, np.pi, 360, endpoint=False), n, 47.5),
        47.5, angles=np.linspace(0, np.pi, 360, endpoint=False),
        apply_log=False)
    img = phantom.phantom_image(params, n)
    inside = img > 0
    assert np.median(rec[inside]) == pytest.approx(mu / n, rel=0.05)


def test_phantom_seeded():
    a, ang, p = phantom.ellipse_sinogram(5, 30, 64, 31.5)
    b, _, q = phantom.ellipse_sinogram(5, 30, 64, 31.5)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(p, q)
    assert a.dtype == np.float32 and a.shape == (30, 64)
    assert np.all(np.isfinite(a))


def test_dropin_validation_before_device():
    """Argument errors of the reference are raised before any device use."""
    from algotom_b200.rec import reconstruction as R
    s = np.ones((10, 20), np.float32)
    with pytest.raises(ValueError, match="Center"):
        R.fbp_reconstruction(s, -1, apply_log=False)
    with pytest.raises(ValueError, match="Center"):
        R.bpf_reconstruction(s, 20, apply_log=False)
    with pytest.raises(ValueError, match="Number of angles"):
        R.fbp_reconstruction(s, 10, angles=np.zeros(7), apply_log=False)
    with pytest.raises(ValueError):
        R.fbp_reconstruction(np.ones(5), 1, apply_log=False)


def test_dropin_mask_and_scale_helpers():
    from algotom_b200.rec import reconstruction as R
    assert R._mask_r2(None, 10, 20) < 0
    assert R._mask_r2(1.0, 10, 20) == 100.0
    # ratio 0: largest disc inside the centred field
    assert R._mask_r2(0.0, 7.0, 20) == pytest.approx((0.7 * 10) ** 2)
    assert R._scale(181) == pytest.approx(np.pi / 180, rel=1e-7)


def test_autotuner_picks_fastest_and_caches(tmp_path):
    from algotom_b200.rec import autotune as AT
    path = tmp_path / "tune.json"
    t = AT.Autotuner(str(path))
    calls = []

    def run(v):
        calls.append(v)
        return {0: 2.0, 1: 1.0}[v]
    key = AT.Autotuner.key("single", "gpu", ncol=1000, nrow=900)
    assert key == AT.Autotuner.key("single", "gpu", ncol=1024, nrow=1000)
    assert t.choose(key, (0, 1), run) == 1
    assert calls == [0, 1]
    assert t.choose(key, (0, 1), run) == 1 and calls == [0, 1]  # cached
    t2 = AT.Autotuner(str(path))  # persisted
    assert t2.choose(key, (0, 1), lambda v: 1 / 0) == 1


def test_autotuner_survives_corrupt_cache(tmp_path):
    from algotom_b200.rec import autotune as AT
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    with pytest.warns(UserWarning, match="unreadable"):
        t = AT.Autotuner(str(path))
    assert t.table == {}
    assert t.choose("k", (0, 1), lambda v: [3.0, 1.0][v]) == 1
    import json
    assert json.loads(path.read_text())["k"]["choice"] == 1


def test_stream_slab_spans_cover_the_stack():
    """Slabs of a host stack streamed through the device: contiguous, cover
    every slice once, at most ``slab`` slices, ramped at both ends of long
    stacks."""
    from algotom_b200.rec.reconstruction import _slab_spans
    for n in (1, 5, 31, 32, 33, 64, 79, 100, 128, 256, 257, 2160):
        for slab in (1, 4, 32):
            sp = _slab_spans(n, slab)
            assert sp[0][0] == 0 and sum(c for _, c in sp) == n
            assert all(0 < c <= slab for _, c in sp)
            assert all(a + c == b for (a, c), (b, _) in zip(sp, sp[1:]))
    sizes = [c for _, c in _slab_spans(256, 32)]
    assert sizes[:3] == [8, 8, 16] and sizes[-3:] == [16, 8, 8]
