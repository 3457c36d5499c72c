"""The 2-D circular ramp filter of BPF (``atb_bpf_filter2d``).

Reference: ``apply_circular_ramp_filter`` (algotom/rec/reconstruction.py
:527-560) and its use in ``bpf_reconstruction`` (:675-684).  The CPU tests
hold the host-built spectrum (exact length and the embedded longer length)
to the oracle's filter through a NumPy model of the device pipeline, and the
transform-length rule of the library.  The GPU tests hold the library's
filter to the FP64 oracle, its padding (numpy's ten modes, corners
included) to ``np.pad``, and BPF at the benchmark slice size.
"""
from unittest import mock

import numpy as np
import pytest

from algotom_b200 import _native as nat
from algotom_b200 import phantom
from algotom_b200.rec import reconstruction as R
from oracle import cpu_port
from oracle import fbp_oracle as O

MODES = ["edge", "constant", "reflect", "symmetric", "wrap", "linear_ramp",
         "mean", "maximum", "minimum", "median"]


def _length(ncol, pad):
    return nat.load().atb_bpf_filter2d_length(ncol, pad)


def test_transform_length_rule():
    """T = N when N's primes are <= 13, else the smallest 7-smooth
    M >= N + ncol - 1; too long is rejected."""
    assert _length(2560, 150) == 2860          # 4 5 11 13
    assert _length(1024, 150) == 2352          # 1324 = 4 331 -> >= 2347
    assert _length(96, 14) == 224              # 124 = 4 31 -> >= 219
    assert _length(65, 9) == 147               # 83 prime -> >= 147 = 3 7^2
    assert _length(2048, 150) == 4410          # 2348 = 4 587 -> >= 4395
    assert _length(4096, 150) == -3            # 4396 -> >= 8491 > 7168
    assert "7168" in nat.last_error()
    assert nat.load().atb_bpf_filter2d_workspace(2560, 150, 2) == \
        2 * 2860 * 2860 * 16 + ((4 * (2 * 2560 + 1) * 8 + 255) // 256) * 256


def _model(imgs, ncol, pad, mode, ramp_win=None, filter_name="hann"):
    """NumPy model of the device pipeline with the host-built spectrum:
    pad, place on the T x T torus, transform, product, inverse, crop; two
    images as one complex image."""
    import torch
    fake = mock.MagicMock()
    fake.call.side_effect = lambda name, *a: _length(*a)
    with mock.patch.object(R, "nat", fake):
        spec, cplx, tw, t = R._circular_spectrum(ramp_win, filter_name, ncol,
                                                 pad, torch.device("cpu"))
    s = spec.numpy().T
    n = ncol + 2 * pad
    z = np.zeros((t, t), complex)
    z[:n, :n] = (np.pad(imgs[0].astype(np.float64), pad, mode=mode)
                 + 1j * np.pad(imgs[1].astype(np.float64), pad, mode=mode))
    y = np.fft.ifft2(np.fft.fft2(z) * s) * t * t
    c = y[pad:pad + ncol, pad:pad + ncol]
    return c.real, c.imag, t


@pytest.mark.parametrize("ncol,pad,mode", [(96, 14, "edge"), (65, 9, "edge"),
                                           (64, 9, "reflect"),
                                           (40, 6, "linear_ramp"),
                                           (128, 19, "median"), (110, 20, "wrap"),
                                           (50, 0, "edge")])
def test_spectrum_reproduces_reference_filter(ncol, pad, mode):
    rng = np.random.default_rng(ncol + pad)
    a = rng.standard_normal((ncol, ncol)).cumsum(0).cumsum(1)
    b = rng.standard_normal((ncol, ncol))
    ea, eb, t = _model((a, b), ncol, pad, mode)
    assert O.rel_l2(ea, O.apply_circular_ramp_filter(a, None, "hann", pad,
                                                      mode)) < 1e-12
    assert O.rel_l2(eb, O.apply_circular_ramp_filter(b, None, "hann", pad,
                                                      mode)) < 1e-12


def _shift_window(n, sy, sx):
    """Circular window whose filter is a circular shift by (sy, sx): the
    crop then shows the padded border of the image."""
    k = np.fft.fftfreq(n) * n
    h = np.exp(-2j * np.pi * (k[:, None] * sy + k[None, :] * sx) / n)
    return np.fft.fftshift(h)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
def test_device_padding_matches_numpy(cuda, mode):
    """The padding inside the filter equals ``np.pad(rec_img, pad, mode)``
    (reconstruction.py:549) for numpy's ten modes, pads wider than the
    image and the corners of the ramp and statistic modes included: a
    window that shifts by +-pad puts the padded border into the crop."""
    rng = np.random.default_rng(2)
    for n in (1, 2, 5, 8, 33):
        x = rng.standard_normal((n, n)).astype(np.float32)
        for pad in (1, 3, 11):
            if mode == "linear_ramp" and pad == 0:
                continue
            p = np.pad(x.astype(np.float64), pad, mode=mode)
            nn = n + 2 * pad
            for sy, sx in ((pad, pad), (-pad, -pad), (pad, -pad)):
                got = R.apply_circular_ramp_filter(
                    x, _shift_window(nn, sy, sx), None, pad, mode)
                ref = np.roll(p, (sy, sx), axis=(0, 1))[pad:pad + n,
                                                        pad:pad + n]
                np.testing.assert_allclose(got, ref.astype(np.float32),
                                           rtol=1e-6, atol=1e-6,
                                           err_msg="%d %d %d %d" % (n, pad,
                                                                    sy, sx))


@pytest.mark.gpu
@pytest.mark.parametrize("ncol,pad,mode,name", [
    (96, 14, "edge", "hann"), (65, 9, "edge", "hann"),
    (128, 19, "reflect", "hamming"), (200, 30, "mean", None),
    (1024, 150, "edge", "hann"), (2560, 150, "edge", "hann")])
def test_filter_matches_fp64_oracle(cuda, ncol, pad, mode, name):
    """Smooth back-projection-like images (where the ramp amplifies
    rounding most), one exact-length and several embedded lengths."""
    rng = np.random.default_rng(ncol)
    img = rng.standard_normal((ncol, ncol)).cumsum(0).cumsum(1)
    img = (img / np.abs(img).max()).astype(np.float32)
    got = R.apply_circular_ramp_filter(img, None, name, pad, mode)
    assert got.dtype == np.float64
    ref = O.apply_circular_ramp_filter(img.astype(np.float64), None, name,
                                       pad, mode)
    assert O.rel_l2(got, ref) < 1e-6


@pytest.mark.gpu
def test_filter_stack_pairs_and_odd_count(cuda):
    """Slices travel in pairs (real and imaginary part); an odd count
    leaves the last one alone; strided [y][slice][x] layout in and out."""
    import torch
    rng = np.random.default_rng(9)
    ncol, nslice = 96, 5
    st = rng.standard_normal((ncol, nslice, ncol)).cumsum(0).astype(np.float32)
    t = torch.from_numpy(st).cuda()
    got = R._circular_filter(t, None, "hann", 14, "edge", mask_r2=-1.0,
                             scale=2.0).cpu().numpy()
    for k in range(nslice):
        ref = 2.0 * O.apply_circular_ramp_filter(st[:, k].astype(np.float64),
                                                 None, "hann", 14, "edge")
        assert O.rel_l2(got[:, k], ref) < 1e-6, k


@pytest.mark.gpu
def test_bpf_full_size_slice(cuda):
    """One 2560^2 slice from 1801 angles through bpf_reconstruction
    against the FP64 oracle (C FP64 back-projector with edge padding +
    the oracle's 2-D filter), at the 1e-5 bar."""
    ncol, nrow, cen = 2560, 1801, 1278.3
    s, ang, _ = phantom.ellipse_sinogram(2000, nrow, ncol, cen, photons=5e3)
    got = R.bpf_reconstruction(s, cen, angles=ang, apply_log=False)
    bp = cpu_port.back_projection(s, ang, cen, edge_pad=True, ref_arith=False)
    ref = O.apply_circular_ramp_filter(bp, None, "hann", 150, "edge")
    ref = ref * O.make_circle_mask(ncol, 1.0) * (np.pi / (nrow - 1))
    err = O.rel_l2(got, ref)
    assert err < 1e-5, err
