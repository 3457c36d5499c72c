"""The oracle against the reference's own outputs (golden vectors).

The vectors in tests/golden were produced by running algotom 1.6.0 itself
(tests/golden/make_golden.py, single-threaded Numba); these tests pin the FP64
restatement (oracle/fbp_oracle.py) and the C restatement (oracle/bp_port.c)
to them, so the oracle can then judge the CUDA path.
"""
import numpy as np
import pytest

from oracle import cpu_port
from oracle import fbp_oracle as O

WINDOWS = ["hann", "bartlett", "blackman", "hamming", "nuttall", "parzen",
           "triang", None]
PAD_MODES = ["edge", "constant", "reflect", "symmetric", "wrap",
             "linear_ramp", "mean", "maximum", "minimum", "median"]


def test_windows_match_reference(golden):
    g = golden("windows")
    for w in (64, 65):
        for name in WINDOWS:
            np.testing.assert_array_equal(
                O.make_smoothing_window(name, w), g["smooth__%s__%d" % (name, w)])
            np.testing.assert_allclose(
                O.make_2d_ramp_window(2, w, name),
                g["ramp2d__%s__%d" % (name, w)], rtol=0, atol=1e-15)
        for name in ("hann", None):
            np.testing.assert_allclose(
                O.make_circular_ramp_window(w, name),
                g["circ__%s__%d" % (name, w)], rtol=0, atol=1e-14)
    for w, ratio in ((65, 1.0), (64, 0.7), (97, 0.93)):
        np.testing.assert_array_equal(O.make_circle_mask(w, ratio),
                                      g["mask__%d__%s" % (w, ratio)])


@pytest.mark.parametrize("mode", PAD_MODES)
def test_filter_pad_modes(golden, mode):
    g = golden("filter")
    ref = g["filt__%s__hann__None" % mode]
    got = O.apply_ramp_filter(g["sino"], None, "hann", None, mode)
    assert O.rel_l2(got, ref) < 1e-6


@pytest.mark.parametrize("name", WINDOWS)
def test_filter_windows(golden, name):
    g = golden("filter")
    ref = g["filt__edge__%s__None" % name]
    got = O.apply_ramp_filter(g["sino"], None, name, None, "edge")
    assert O.rel_l2(got, ref) < 1e-6


@pytest.mark.parametrize("pad", [0, 7, 200])
@pytest.mark.parametrize("mode", ["edge", "reflect", "wrap"])
def test_filter_pads(golden, pad, mode):
    g = golden("filter")
    got = O.apply_ramp_filter(g["sino"], None, "hann", pad, mode)
    assert O.rel_l2(got, g["filt__%s__hann__%d" % (mode, pad)]) < 1e-6


def test_filter_odd_width(golden):
    g = golden("filter")
    got = O.apply_ramp_filter(g["sino_odd"], None, "hann", None, "edge")
    assert O.rel_l2(got, g["filtodd__edge__hann__None"]) < 1e-6


def test_filter_convolution_form():
    """apply_ramp_filter is a circular convolution with filter_kernel_spatial."""
    rng = np.random.default_rng(3)
    ncol, pad = 40, 9
    n = ncol + 2 * pad
    x = rng.standard_normal((2, ncol))
    k = O.filter_kernel_spatial(n, "hann")
    xp = np.pad(x, ((0, 0), (pad, pad)), mode="edge")
    conv = np.array([[sum(xp[r, m] * k[(j - m) % n] for m in range(n))
                      for j in range(pad, pad + ncol)] for r in range(2)])
    np.testing.assert_allclose(conv, O.apply_ramp_filter(x, None, "hann", pad),
                               atol=1e-14)


@pytest.mark.parametrize("cen", [47.5, 45.3, 52.0])
@pytest.mark.parametrize("ep", [0, 1])
def test_backprojection(golden, cen, ep):
    g = golden("bp")
    ref = g["bp__%s__%d" % (cen, ep)]
    got = O.back_projection(g["filtered"], g["angles"], cen, bool(ep))
    # the reference accumulates in float32 with float32 trig
    assert O.rel_l2(got, ref) < 1e-6


@pytest.mark.parametrize("ep", [0, 1])
def test_backprojection_odd_360(golden, ep):
    g = golden("bp")
    got = O.back_projection(g["filtered_odd"], g["angles_odd"], 40.0, bool(ep))
    assert O.rel_l2(got, g["bpodd__40.0__%d" % ep]) < 1e-6


@pytest.mark.parametrize("cen", [47.5, 45.3, 52.0])
@pytest.mark.parametrize("ep", [0, 1])
def test_c_port_bit_exact(golden, cen, ep):
    """The C restatement reproduces the single-threaded reference bit for bit."""
    g = golden("bp")
    got = cpu_port.back_projection(g["filtered"], g["angles"], cen, bool(ep),
                                   ref_arith=True, nthreads=3)
    np.testing.assert_array_equal(got, g["bp__%s__%d" % (cen, ep)])
    f64 = cpu_port.back_projection(g["filtered"], g["angles"], cen, bool(ep),
                                   ref_arith=False)
    assert O.rel_l2(f64, O.back_projection(g["filtered"], g["angles"], cen,
                                           bool(ep))) < 1e-12


def _recon_cases():
    return [("fbp", O.fbp_reconstruction), ("bpf", O.bpf_reconstruction)]


@pytest.mark.parametrize("name,fn", _recon_cases())
def test_drivers_2d(golden, name, fn):
    g = golden("recon")
    sino, ang = g["sino"], g["angles"]
    tol = 1e-5 if name == "bpf" else 2e-6
    for ratio in (1.0, 0.0, None):
        got = fn(sino, 47.5, angles=ang, ratio=ratio, apply_log=False)
        assert O.rel_l2(got, g["%s__2d__%s" % (name, ratio)]) < tol
    got = fn(sino, 45.3, apply_log=False)
    assert O.rel_l2(got, g["%s__2d__defang" % name]) < tol
    got = fn(sino, 47.5, angles=ang, filter_name=None, pad=10,
             pad_mode="reflect", apply_log=False)
    # BPF without a smoothing window: the reference's complex64 fft2 of the
    # (very smooth) back-projected image leaves white rounding noise that
    # the bare ramp amplifies to ~1e-5 of the result
    tol_nf = 5e-5 if name == "bpf" else tol
    assert O.rel_l2(got, g["%s__2d__nofilter__reflect" % name]) < tol_nf
    got = fn(g["trans"], 47.5, angles=ang, apply_log=True)
    assert O.rel_l2(got, g["%s__2d__log" % name]) < tol


@pytest.mark.parametrize("name,fn", _recon_cases())
def test_drivers_3d(golden, name, fn):
    g = golden("recon")
    tol = 1e-5 if name == "bpf" else 2e-6
    got = fn(g["s3"], 47.5, angles=g["angles"], ratio=0.0, apply_log=False)
    assert got.shape == (96, 3, 96)
    assert O.rel_l2(got, g["%s__3d__0.0" % name]) < tol
    got = fn(g["s3"][:, :1], 47.5, angles=g["angles"], apply_log=False)
    assert got.shape == (96, 1, 96)
    assert O.rel_l2(got, g["%s__3d1__1.0" % name]) < tol


def test_reference_unittest_fixture(golden):
    """The reference's own unit-test phantom (test_reconstruction.py:50-65)."""
    g = golden("unittest")
    s180 = g["sino_360"][:37]
    fbp = O.fbp_reconstruction(s180, 32, apply_log=False)
    assert O.rel_l2(fbp, g["fbp_180"]) < 2e-6
    assert np.median(np.abs(g["mat"] - fbp)) <= 0.2
    bpf = O.bpf_reconstruction(s180, 32, apply_log=False)
    assert O.rel_l2(bpf, g["bpf_180"]) < 1e-5


def test_validation_errors():
    s = np.ones((10, 20), np.float32)
    with pytest.raises(ValueError):
        O.fbp_reconstruction(s, -1, apply_log=False)
    with pytest.raises(ValueError):
        O.fbp_reconstruction(s, 10, angles=np.zeros(7), apply_log=False)
