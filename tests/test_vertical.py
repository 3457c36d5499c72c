"""Vertical-slice reconstruction (algotom/rec/vertrec.py).

CPU tests pin the FP64 oracle (``oracle/vertical_oracle.py``) and the host
slice geometry to vectors produced by the reference's CPU path
(``tests/golden/golden_vertical.npz``), and check the device-side FP64
row padding and "after" filter against NumPy.  GPU tests hold the device
path, through the C ABI, to the reference's outputs and to the oracle:

- back-projectors: 1e-6 relative L2 (the reference accumulates in float32);
- reconstructions: 1e-5 relative L2 (the "after" ramp filter of the
  reference runs a float32 forward FFT: ~1e-6 from FP64 at these sizes);
- the slice geometry: bit-exact;
- warnings, in-place repair of values <= 0, argument errors, output dtypes:
  as the reference.
"""
import warnings

import numpy as np
import pytest

from algotom_b200 import _native as nat
from oracle import fbp_oracle as O
from oracle import vertical_oracle as V

LINES = ((32, 0.0), (20, 30.0), (40, 60.0), (10, 90.0), (50, 150.0))
TOL_BP = 1e-6
TOL = 1e-5
PAD_MODES = ["edge", "constant", "reflect", "symmetric", "wrap",
             "linear_ramp", "mean", "maximum", "minimum", "median"]


def _pts_keys(g):
    for k in g.files:
        if k.startswith("pts__") and k.endswith("__x"):
            _, w, idx, alpha, _ = k.split("__")
            yield k, int(w), int(idx), float(alpha)


# ------------------------------------------------------------- CPU
def test_geometry_bit_exact(golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    n = 0
    for k, w, idx, alpha in _pts_keys(g):
        for fn in (VR._get_points_single_line, V.points_single_line):
            xs, ys = fn(idx, alpha, w)
            assert np.array_equal(xs, g[k]) and np.array_equal(
                ys, g[k[:-1] + "y"]), (fn, k)
        n += 1
    assert n == 24
    xm, ym = VR._get_points_multiple_lines(20, 44, 45.0, 64, 8)
    assert xm.dtype == np.float32
    assert np.array_equal(xm, g["xm"]) and np.array_equal(ym, g["ym"])


def test_geometry_errors():
    from algotom_b200.rec import vertrec as VR
    with pytest.raises(ValueError, match="Angle is out of range"):
        VR._get_points_single_line(3, 181.0, 16)
    with pytest.raises(ValueError, match="Slice index is out of range"):
        VR._get_points_single_line(16, 10.0, 16)


@pytest.mark.parametrize("idx,alpha", LINES)
def test_oracle_back_projection(golden, idx, alpha):
    g = golden("vertical")
    xs, ys = V.points_single_line(idx, alpha, 64)
    for ep in (False, True):
        got = V.vertical_back_projection(g["att"], g["angles"], xs, ys,
                                         float(g["center"]), ep)
        assert O.rel_l2(got, g["vbp__%d__%s__%s" % (idx, alpha, ep)]) < \
            TOL_BP


def test_oracle_reconstructions(golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    tr, ang, cen = g["trans"], g["angles"], float(g["center"])
    xs, ys = V.points_single_line(30, 0.0, 64)
    for name, kw in (("after", {}), ("before", {"ramp_filter": "before"}),
                     ("none", {"ramp_filter": None})):
        got = V.vertical_reconstruction(tr, [xs], [ys], cen, angles=ang,
                                        **kw)[0]
        assert O.rel_l2(got, g["vrec__" + name]) < TOL
    xm, ym = VR._get_points_multiple_lines(20, 40, 45.0, 64, 5)
    got = V.vertical_reconstruction(tr, xm, ym, cen, angles=ang)
    assert O.rel_l2(got, g["vrec_multi"]) < TOL
    xm, ym = VR._get_points_multiple_lines_different_angles(
        [10, 30, 50], [0.0, 60.0, 120.0], 64)
    got = V.vertical_reconstruction(tr, xm, ym, cen, angles=ang,
                                    ramp_filter="before", masking=True)
    assert O.rel_l2(got, g["vrec_diff"]) < TOL


@pytest.mark.parametrize("mode", PAD_MODES)
def test_row_padding_matches_numpy(mode):
    import torch
    from algotom_b200.rec.padding import pad_rows
    rng = np.random.default_rng(1)
    for n in (1, 2, 3, 7, 8):
        x = rng.standard_normal((3, n))
        for pad in (0, 1, 4, 19):
            got = pad_rows(torch.from_numpy(x), pad, mode).numpy()
            ref = np.pad(x, ((0, 0), (pad, pad)), mode=mode)
            if mode == "mean":  # summation order differs from NumPy's
                assert np.allclose(got, ref, rtol=1e-15, atol=1e-15)
            else:
                assert np.array_equal(got, ref), (n, pad)


@pytest.mark.gpu
def test_fp64_after_filter_matches_oracle(cuda):
    """The after filter of large smooth FP64 sums (the ramp removes their
    mean) against the oracle's, 40 + 12 = 52 = 4 x 13 points; equal rows
    give bit-equal results, as NumPy's do (the centre search normalises by
    a maximum that such rows reach exactly)."""
    import torch
    from algotom_b200.rec import vertrec as VR
    rng = np.random.default_rng(2)
    x = 50.0 + rng.standard_normal((2, 3, 40)).cumsum(axis=2)
    x[1, 2] = x[1, 1] = x[0, 0]
    got = VR._after_filter64(torch.from_numpy(x).to(cuda), "hann", 6,
                             "edge").cpu().numpy()
    ref = np.stack([V.ver_ramp_filter(v, "hann", 6, "edge") for v in x])
    assert np.max(np.abs(got - ref)) < 1e-12 * np.max(np.abs(x))
    assert np.array_equal(got[1, 2], got[0, 0])
    assert np.array_equal(got[1, 1], got[0, 0])


def test_abi_argument_errors():
    lib = nat.load()
    one = 1
    assert lib.atb_vertical_backproject(None, 8, 8, 2, 2, 8, one, one, 8, 8,
                                        1, 3.0, None, 0, one, 8, 8, None, 0,
                                        None) == -1
    assert lib.atb_vertical_backproject(one, 8, 8, 0, 2, 8, one, one, 8, 8,
                                        1, 3.0, None, 0, one, 8, 8, None, 0,
                                        None) == -1
    assert lib.atb_vertical_backproject(one, 8, 8, 2, 2, 8, one, one, 8, 8,
                                        1, float("nan"), None, 0, one, 8, 8,
                                        None, 0, None) == -1
    assert lib.atb_vertical_backproject(one, 1 << 31, 1 << 30, 2, 4, 8, one,
                                        one, 8, 8, 1, 3.0, None, 0, one, 8,
                                        8, None, 0, None) == -3
    # a small output asks for scratch to split the angles, a large one not
    assert lib.atb_vertical_workspace(1801, 64, 2560, 1) > 0
    assert lib.atb_vertical_workspace(1801, 2048, 2560, 64) == 0
    assert lib.atb_vertical_workspace(0, 64, 2560, 1) == 0
    assert lib.atb_flat_log(one, 0, 8, 8, 1, 1, 8, one, None, 8, 1, one, 8,
                            8, one, None) == -1  # dark without flat_dark
    assert lib.atb_flat_log(one, 7, 8, 8, 1, 1, 8, None, None, 8, 1, one, 8,
                            8, one, None) == -1  # unknown dtype
    assert b"dtype" in lib.atb_last_error()


def test_reconstruction_argument_errors():
    from algotom_b200.rec import vertrec as VR
    p = np.ones((5, 4, 8), np.float32)
    with pytest.raises(ValueError, match="Must use one of these options"):
        VR.vertical_reconstruction(p, 3, 3.0, ramp_filter="middle")
    with pytest.raises(ValueError, match="Wrong value of proj_start"):
        VR.vertical_reconstruction(p, 3, 3.0, proj_start=5)
    with pytest.raises(ValueError, match="Number of angles"):
        VR.vertical_reconstruction(p, 3, 3.0, angles=np.zeros(4))
    with pytest.raises(ValueError, match="Can't crop"):
        VR.vertical_reconstruction(p, 3, 3.0, crop=(2, 2, 0, 0))
    with pytest.raises(ValueError, match="Center"):
        VR.vertical_reconstruction(p, 3, 7.5)
    with pytest.raises(ValueError, match="Index"):
        VR.vertical_reconstruction(p, 8, 3.0)
    with pytest.raises(ValueError, match="Start index"):
        VR.vertical_reconstruction_multiple(p, 2, 9, 3.0)
    with pytest.raises(ValueError, match="Number of slice indices"):
        VR.vertical_reconstruction_different_angles(p, [1, 2], [0.0], 3.0)
    with pytest.raises(ValueError, match="Slice index"):
        VR.vertical_reconstruction_different_angles(p, [1, 9], [0.0, 1.0],
                                                    3.0)


# ------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("idx,alpha", LINES)
def test_back_projection_cpu_form(cuda, golden, idx, alpha):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    xs, ys = V.points_single_line(idx, alpha, 64)
    for ep in (False, True):
        got = VR.vertical_back_projection_cpu(g["att"], g["angles"], xs, ys,
                                              float(g["center"]), ep)
        assert got.dtype == np.float32 and got.shape == (10, 64)
        ref = g["vbp__%d__%s__%s" % (idx, alpha, ep)]
        assert O.rel_l2(got, ref) < TOL_BP
        ora = V.vertical_back_projection(g["att"], g["angles"], xs, ys,
                                         float(g["center"]), ep)
        assert O.rel_l2(got, ora) < TOL_BP


@pytest.mark.gpu
def test_back_projection_gpu_and_chunk_forms(cuda, golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    att, ang, cen = g["att"], g["angles"], float(g["center"])
    xs, ys = V.points_single_line(20, 30.0, 64)
    got = VR.vertical_back_projection_gpu(att, ang, xs, ys, cen)
    # float32-rounded inputs, as the reference's GPU kernel receives them
    ora = V.vertical_back_projection(
        att, np.float32(ang).astype(np.float64),
        np.float32(xs).astype(np.float64), np.float32(ys).astype(np.float64),
        float(np.float32(cen)))
    assert O.rel_l2(got, ora) < TOL_BP
    for ep in (False, True):
        got = VR.vertical_back_projection_cpu_chunk(att, ang, g["xm"],
                                                    g["ym"], cen, ep)
        assert got.shape == (4, 10, 64)
        assert O.rel_l2(got, g["vbpchunk__%s" % ep]) < TOL_BP
        got = VR.vertical_back_projection_gpu_chunk(att, ang, g["xm"],
                                                    g["ym"], cen, ep)
        assert O.rel_l2(got, g["vbpchunk__%s" % ep]) < 1e-5


@pytest.mark.gpu
def test_back_projection_many_rows_and_points(cuda):
    """Heights and widths across the kernel's 32-row / 64-point blocks and
    more than one 32-angle table."""
    from algotom_b200.rec import vertrec as VR
    rng = np.random.default_rng(3)
    for depth, height, width in ((37, 70, 130), (5, 1, 3), (65, 33, 64)):
        p = rng.standard_normal((depth, height, width)).astype(np.float32)
        ang = np.linspace(0, np.pi, depth)
        cen = 0.5 * (width - 1) + 0.3
        xs, ys = V.points_single_line(width // 3, 25.0, width)
        for ep in (False, True):
            got = VR.vertical_back_projection_cpu(p, ang, xs, ys, cen, ep)
            ref = V.vertical_back_projection(p, ang, xs, ys, cen, ep)
            assert O.rel_l2(got, ref) < TOL_BP


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["after", "before", "none", "crop_range",
                                  "flat", "alpha"])
def test_vertical_reconstruction_matches_reference(cuda, golden, name):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    cen = float(g["center"])
    kw = {"after": dict(), "before": dict(ramp_filter="before"),
          "none": dict(ramp_filter=None),
          "crop_range": dict(crop=(1, 2, 3, 4), proj_start=2, proj_stop=70,
                             chunk_size=16, masking=True),
          "flat": dict(flat_field=g["flat"], dark_field=g["dark"],
                       chunk_size=20, ramp_filter="before", pad=10,
                       pad_mode="reflect"),
          "alpha": dict(alpha=70.0, filter_name="hamming",
                        chunk_size=None)}[name]
    src = g["raw"] if "flat_field" in kw else g["trans"]
    ang = g["angles"][2:70] if "proj_stop" in kw else g["angles"]
    c = cen - (3 if "crop" in kw else 0)
    ref = g["vrec__" + name]
    for gpu in (False, True):
        got = VR.vertical_reconstruction(src.copy(), 30, c, angles=ang,
                                         gpu=gpu, show_progress=False, **kw)
        assert got.dtype == ref.dtype and got.shape == ref.shape
        assert O.rel_l2(got, ref) < TOL, gpu


@pytest.mark.gpu
def test_multiple_and_different_angles(cuda, golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    cen, ang = float(g["center"]), g["angles"]
    got = VR.vertical_reconstruction_multiple(
        g["trans"].copy(), 20, 40, cen, alpha=45.0, step_index=5, angles=ang,
        chunk_size=25, gpu=False, show_progress=False)
    assert got.dtype == np.float32 and got.shape == (5, 10, 64)
    assert O.rel_l2(got, g["vrec_multi"]) < TOL
    got = VR.vertical_reconstruction_different_angles(
        g["trans"].copy(), [10, 30, 50], [0.0, 60.0, 120.0], cen, angles=ang,
        ramp_filter="before", chunk_size=30, masking=True, gpu=False,
        show_progress=False)
    assert O.rel_l2(got, g["vrec_diff"]) < TOL


@pytest.mark.gpu
def test_log_warnings_and_repair(cuda, golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    bad = g["trans"].copy()
    bad[5, 3, 7] = 0.0
    bad[40, 8, 20] = -1.0
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        got = VR.vertical_reconstruction(bad, 30, float(g["center"]),
                                         angles=g["angles"], chunk_size=30,
                                         gpu=False, show_progress=False)
    msgs = [str(w.message) for w in caught if "logarithm" in str(w.message)]
    assert msgs == list(g["vrec_log_warnings"])
    assert np.array_equal(bad, g["vrec_log_mutated"])
    assert O.rel_l2(got, g["vrec_log"]) < TOL


@pytest.mark.gpu
def test_device_pinned_and_uint16_inputs(cuda, golden):
    import torch
    from algotom_b200.rec import vertrec as VR
    g = golden("vertical")
    cen, ang = float(g["center"]), g["angles"]
    ref = VR.vertical_reconstruction(g["trans"].copy(), 30, cen, angles=ang,
                                     gpu=False, show_progress=False)
    t = torch.as_tensor(g["trans"], device="cuda")
    got = VR.vertical_reconstruction(t, 30, cen, angles=ang, gpu=False,
                                     show_progress=False)
    assert isinstance(got, torch.Tensor) and got.is_cuda
    assert np.allclose(got.cpu().numpy(), ref, rtol=0, atol=1e-9)
    # pinned host memory (direct strided copies), cropped and whole
    pin = torch.empty(g["trans"].shape, dtype=torch.float32,
                      pin_memory=True)
    pin.copy_(torch.from_numpy(g["trans"]))
    got = VR.vertical_reconstruction(pin.numpy(), 30, cen, angles=ang,
                                     gpu=False, show_progress=False,
                                     chunk_size=7)
    assert np.allclose(got, ref, rtol=0, atol=1e-9)
    got = VR.vertical_reconstruction(pin.numpy(), 30, cen - 3,
                                     angles=ang[2:70], crop=(1, 2, 3, 4),
                                     proj_start=2, proj_stop=70,
                                     chunk_size=16, masking=True, gpu=False,
                                     show_progress=False)
    assert O.rel_l2(got, g["vrec__crop_range"]) < TOL
    # raw uint16 counts with flat / dark fields
    counts = np.round(g["raw"] * 4000).astype(np.uint16)
    flat, dark = g["flat"] * 4000, g["dark"] * 4000
    got = VR.vertical_reconstruction(counts, 30, cen, angles=ang,
                                     flat_field=flat, dark_field=dark,
                                     gpu=False, show_progress=False)
    xs, ys = V.points_single_line(30, 0.0, 64)
    ora = V.vertical_reconstruction(counts.astype(np.float32), [xs], [ys],
                                    cen, angles=ang, flat_field=flat,
                                    dark_field=dark)[0]
    assert O.rel_l2(got, ora) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["edge", "reflect", "constant", "wrap",
                                  "linear_ramp", "mean", "median"])
@pytest.mark.parametrize("width,pad", [(96, 14), (130, 10), (63, 6), (1, 0),
                                       (2, 0), (3, 1)])
def test_after_filter64_matches_numpy(cuda, mode, width, pad):
    """The FP64 after filter (atb_filter_rows64) against the reference's
    numpy expression (vertrec.py:677-684) at an embedded transform length
    (96 + 28 = 124 = 4 x 31 is not 13-smooth: 224), at the padded width
    itself (130 + 20 = 150), both even (real transforms of half length), and
    at an odd one (63 + 12 = 75: one complex transform per row), and at the
    smallest widths (transforms of 1, 2 and 5 points, plans of zero or one
    stage), for index, ramp and statistic pad modes; two slices of an odd
    row count."""
    import torch
    from algotom_b200.rec import vertrec as VR
    from algotom_b200.rec import windows as W
    rng = np.random.default_rng(width + pad)
    ver = rng.standard_normal((2, 7, width))
    got = VR._after_filter64(torch.as_tensor(ver, device="cuda"), "hann",
                             pad, mode).cpu().numpy()
    n = width + 2 * pad
    win = np.abs(W.ramp_window_row(n, "hann"))
    for k in range(2):
        xp = np.pad(ver[k], ((0, 0), (pad, pad)), mode=mode)
        ref = np.real(np.fft.ifft(np.fft.ifftshift(
            np.fft.fftshift(np.fft.fft(xp), axes=1) * win,
            axes=1)))[:, pad:pad + width]
        assert np.abs(got[k] - ref).max() <= 1e-12 * max(np.abs(ref).max(),
                                                         np.abs(ver).max())
