"""Parity of the CUDA path (through the C ABI) with the reference and oracle.

Tolerances: the filter and every FP32 reconstruction must be within 1e-5
relative L2 of the FP64 oracle (the bar this path is held to); against the
reference's own float32 outputs (golden vectors) the same bound applies.
"""
import numpy as np
import pytest
import torch

from algotom_b200 import _native as nat
from algotom_b200 import phantom
from algotom_b200.rec import reconstruction as R
from oracle import cpu_port
from oracle import fbp_oracle as O

pytestmark = pytest.mark.gpu

WINDOWS = ["hann", "bartlett", "blackman", "hamming", "nuttall", "parzen",
           "triang", None]
PAD_MODES = ["edge", "constant", "reflect", "symmetric", "wrap",
             "linear_ramp", "mean", "maximum", "minimum", "median"]
TOL = 1e-5


# ----------------------------------------------------------------- filter
@pytest.mark.parametrize("mode", PAD_MODES)
def test_filter_pad_modes(cuda, golden, mode):
    g = golden("filter")
    got = R.apply_ramp_filter(g["sino"], None, "hann", None, mode)
    assert got.dtype == np.float64 and got.shape == g["sino"].shape
    assert O.rel_l2(got, g["filt__%s__hann__None" % mode]) < 1e-6
    assert O.rel_l2(got, O.apply_ramp_filter(g["sino"], None, "hann", None,
                                             mode)) < 1e-6


@pytest.mark.parametrize("name", WINDOWS)
def test_filter_windows(cuda, golden, name):
    g = golden("filter")
    got = R.apply_ramp_filter(g["sino"], None, name, None, "edge")
    assert O.rel_l2(got, g["filt__edge__%s__None" % name]) < 1e-6


@pytest.mark.parametrize("pad", [0, 7, 200])
@pytest.mark.parametrize("mode", ["edge", "reflect", "wrap"])
def test_filter_pads(cuda, golden, pad, mode):
    g = golden("filter")
    got = R.apply_ramp_filter(g["sino"], None, "hann", pad, mode)
    assert O.rel_l2(got, g["filt__%s__hann__%d" % (mode, pad)]) < 1e-6


def test_filter_odd_and_tiny_rows(cuda, golden):
    g = golden("filter")
    got = R.apply_ramp_filter(g["sino_odd"], None, "hann", None, "edge")
    assert O.rel_l2(got, g["filtodd__edge__hann__None"]) < 1e-6
    rng = np.random.default_rng(0)
    for ncol, nrow in ((1, 3), (2, 1), (5, 7), (3, 2)):
        x = rng.standard_normal((nrow, ncol)).astype(np.float32)
        for mode in ("edge", "reflect", "symmetric", "median"):
            got = R.apply_ramp_filter(x, None, "hann", 4, mode)
            ref = O.apply_ramp_filter(x, None, "hann", 4, mode)
            assert np.abs(got - ref).max() <= 1e-6 * max(1.0, np.abs(ref).max())


def test_filter_per_row_window(cuda):
    """A ramp window that differs per row takes the per-angle path."""
    sino, _, _ = phantom.ellipse_sinogram(3, 20, 64, 31.5)
    n = 64 + 2 * 9
    win = O.make_2d_ramp_window(20, n, "hann")
    win = win * np.linspace(0.5, 1.5, 20)[:, None]
    got = R.apply_ramp_filter(sino, win, None, 9)
    assert O.rel_l2(got, O.apply_ramp_filter(sino, win, None, 9)) < 1e-6
    # a stack with the same per-row window: two slices per transform
    s3 = np.stack([sino, 2 * sino, -sino], axis=1)
    t = torch.from_numpy(s3).cuda()
    f = R.filter_sinograms(t, 9, "edge", False, win, None)
    for k in range(3):
        ref = O.apply_ramp_filter(s3[:, k], win, None, 9)
        assert O.rel_l2(f[:, k].cpu().numpy(), ref) < 1e-6


def test_filter_with_log(cuda):
    sino, _, _ = phantom.ellipse_sinogram(4, 30, 80, 39.5)
    trans = np.exp(-sino).astype(np.float32)
    t = torch.from_numpy(trans[:, None, :]).cuda()
    f = R.filter_sinograms(t, 12, "edge", True, None, "hann")[:, 0]
    ref = O.apply_ramp_filter(-np.log(trans.astype(np.float64)), None,
                              "hann", 12)
    assert O.rel_l2(f.cpu().numpy(), ref) < 1e-6


def test_filter_limits(cuda):
    x = np.zeros((2, 9000), np.float32)
    # N = 9300 = 2^2 3 5^2 31 and N + ncol - 1 > 16384: no exact length
    with pytest.raises(nat.NativeLibraryError, match="16384"):
        R.apply_ramp_filter(x, None, "hann", 150)
    # 8000 columns: length 16384, too long to stage rows in shared memory,
    # so one CTA per row pair reads them from global memory
    x = np.random.default_rng(2).standard_normal((3, 8000)).astype(np.float32)
    got = R.apply_ramp_filter(x, None, "hann", 150)
    assert O.rel_l2(got, O.apply_ramp_filter(x, None, "hann", 150)) < 1e-6


@pytest.mark.parametrize("ncol", [2560, 2557])
def test_filter_persistent_many_pairs(cuda, ncol):
    """The persistent filter at the benchmark's width: many row pairs per
    CTA, the next pair's rows prefetched; 16-byte row copies (2560) and
    4-byte copies (2557, rows not 16-byte aligned), a strided slice view,
    a pair split across two angles (odd slice count); checked rows against
    the FP64 oracle."""
    rng = np.random.default_rng(ncol)
    nrow, nslice = 451, 5
    x = torch.from_numpy(rng.standard_normal((nrow, nslice + 1, ncol))
                         .astype(np.float32)).cuda()[:, 1:, :]  # a view
    f = R.filter_sinograms(x, 150, "edge", False, None, "hann").cpu().numpy()
    xs = x.cpu().numpy()
    for k in (0, 2, 4):
        rows = [0, 1, 226, 449, 450]
        got = f[rows, k, :]
        ref = O.apply_ramp_filter(xs[rows, k, :], None, "hann", 150, "edge")
        assert O.rel_l2(got, ref) < 1e-6


# ---------------------------------------------------------- back-projection
@pytest.mark.parametrize("cen", [47.5, 45.3, 52.0])
@pytest.mark.parametrize("ep", [0, 1])
def test_backprojection_vs_reference(cuda, golden, cen, ep):
    g = golden("bp")
    got = R.back_projection_gpu(g["filtered"], g["angles"], cen,
                                edge_pad=bool(ep))
    assert got.dtype == np.float32 and got.shape == (96, 96)
    oracle = O.back_projection(g["filtered"], g["angles"], cen, bool(ep))
    assert O.rel_l2(got, oracle) < 1e-6
    assert O.rel_l2(got, g["bp__%s__%d" % (cen, ep)]) < TOL


@pytest.mark.parametrize("ep", [0, 1])
def test_backprojection_odd_360(cuda, golden, ep):
    g = golden("bp")
    f, a = g["filtered_odd"], g["angles_odd"]
    got = R.back_projection_gpu(f, a, 40.0, edge_pad=bool(ep))
    assert O.rel_l2(got, O.back_projection(f, a, 40.0, bool(ep))) < 1e-6
    assert O.rel_l2(got, g["bpodd__40.0__%d" % ep]) < TOL


@pytest.mark.parametrize("ncol,nrow,cen", [
    (17, 5, 8.0), (64, 33, 31.5), (65, 64, 0.0), (100, 1, 99.99),
    (130, 97, 64.2), (257, 31, 128.0), (63, 2, 62.0)])
@pytest.mark.parametrize("ep", [0, 1])
def test_backprojection_shapes_and_centres(cuda, ncol, nrow, cen, ep):
    rng = np.random.default_rng(ncol * 7 + nrow)
    s = rng.standard_normal((nrow, ncol)).astype(np.float32)
    ang = np.concatenate([[0.0, np.pi / 2], rng.uniform(-4, 8, nrow)])[:nrow]
    got = R.back_projection_gpu(s, ang, cen, edge_pad=bool(ep))
    ref = O.back_projection(s, ang, cen, bool(ep))
    # white-noise sinograms have neighbour differences as large as the
    # values, so FP32 positions weigh more than on phantom data
    assert O.rel_l2(got, ref) < TOL


def test_backprojection_chunk_and_kahan_modes(cuda):
    rng = np.random.default_rng(11)
    s3 = rng.standard_normal((45, 3, 70)).astype(np.float32)
    ang = np.linspace(0, np.pi, 45)
    got = R.back_projection_gpu_chunk(s3, ang, 34.7)
    assert got.shape == (70, 3, 70)
    t = torch.from_numpy(s3).cuda()
    got2 = R.backproject(t, ang, 34.7, kahan="angle").cpu().numpy()
    for k in range(3):
        ref = O.back_projection(s3[:, k], ang, 34.7)
        assert O.rel_l2(got[:, k], ref) < TOL
        assert O.rel_l2(got2[:, k], ref) < TOL


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16,
                                   torch.bfloat16])
def test_tma_staging_matches_cp_async(cuda, dtype):
    """TMA box loads stage the same detector windows as cp.async: identical
    results for 4-, 2- and 1-slice CTAs, both single-slice tile variants,
    edge padding, per-angle Kahan and the circle mask, with windows that
    reach past both detector edges; no staging wait runs out."""
    nat.call("atb_backproject_status", 1)
    rng = np.random.default_rng(21)
    for ncol, nslice, nrow, cen in ((256, 7, 181, 127.3), (96, 1, 60, 20.0),
                                    (64, 4, 37, 60.5), (32, 2, 19, 3.0),
                                    (520, 3, 93, 300.25)):
        s = rng.standard_normal((nrow, nslice, ncol)).astype(np.float32)
        t = torch.from_numpy(s).to(cuda).to(dtype)
        ang = np.concatenate([[0.0, np.pi / 2], rng.uniform(0, np.pi, nrow)])
        ang = ang[:nrow]
        for kw in (dict(), dict(edge_pad=True), dict(kahan="angle"),
                   dict(variant=1), dict(mask_r2=float((ncol // 3) ** 2))):
            a = R.backproject(t, ang, cen, staging="tma", **kw)
            b = R.backproject(t, ang, cen, staging="cp.async", **kw)
            assert torch.equal(a, b), (ncol, nslice, kw)
        if dtype == torch.float32:
            got = R.backproject(t, ang, cen)[:, 0].cpu().numpy()
            ref = O.back_projection(s[:, 0], ang, cen)
            assert O.rel_l2(got, ref) < TOL
    assert nat.call("atb_backproject_status", 0) == 0


def test_backprojection_deterministic(cuda):
    s, ang, _ = phantom.ellipse_sinogram(8, 181, 300, 149.5)
    t = torch.from_numpy(s).cuda()
    a = R.backproject(t[:, None], ang, 149.5)
    b = R.backproject(t[:, None], ang, 149.5)
    assert torch.equal(a, b)


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_reduced_storage_reports_error(cuda, storage):
    """FP16/BF16 filtered storage: FP32 accumulation, bounded error."""
    s, ang, _ = phantom.ellipse_sinogram(9, 180, 256, 127.5)
    ref = O.fbp_reconstruction(s, 127.5, angles=ang, apply_log=False)
    got = R.fbp_reconstruction(s, 127.5, angles=ang, apply_log=False,
                               storage=storage)
    err = O.rel_l2(got, ref)
    assert err < (2e-3 if storage == "float16" else 1.5e-2)


# ------------------------------------------------------------ FBP and BPF
@pytest.mark.parametrize("name", ["fbp", "bpf"])
def test_recon_2d_vs_reference(cuda, golden, name):
    g = golden("recon")
    fn = R.fbp_reconstruction if name == "fbp" else R.bpf_reconstruction
    dtypes = eval(str(g["dtypes"]))
    sino, ang = g["sino"], g["angles"]
    tol = TOL
    for ratio in (1.0, 0.0, None):
        key = "%s__2d__%s" % (name, ratio)
        got = fn(sino.copy(), 47.5, angles=ang, ratio=ratio, apply_log=False)
        assert str(got.dtype) == dtypes[key]
        assert O.rel_l2(got, g[key]) < tol
    got = fn(sino.copy(), 45.3, apply_log=False)
    assert O.rel_l2(got, g["%s__2d__defang" % name]) < tol
    got = fn(sino.copy(), 47.5, angles=ang, filter_name=None, pad=10,
             pad_mode="reflect", apply_log=False)
    ref_o = (O.fbp_reconstruction if name == "fbp" else O.bpf_reconstruction)(
        sino, 47.5, angles=ang, filter_name=None, pad=10, pad_mode="reflect",
        apply_log=False)
    assert O.rel_l2(got, ref_o) < tol
    t = g["trans"].copy()
    with pytest.warns(UserWarning, match="values <= 0.0"):
        got = fn(t, 47.5, angles=ang, apply_log=True)
    np.testing.assert_array_equal(t, g["%s__2d__log__mutated" % name])
    assert O.rel_l2(got, g["%s__2d__log" % name]) < tol


@pytest.mark.parametrize("name", ["fbp", "bpf"])
def test_recon_3d_vs_reference(cuda, golden, name):
    g = golden("recon")
    fn = R.fbp_reconstruction if name == "fbp" else R.bpf_reconstruction
    tol = TOL
    got = fn(g["s3"].copy(), 47.5, angles=g["angles"], ratio=0.0,
             apply_log=False, ncore=1)
    assert got.shape == (96, 3, 96) and got.dtype == np.float32
    assert O.rel_l2(got, g["%s__3d__0.0" % name]) < tol
    got = fn(g["s3"][:, :1].copy(), 47.5, angles=g["angles"], apply_log=False)
    assert got.shape == (96, 1, 96)
    assert O.rel_l2(got, g["%s__3d1__1.0" % name]) < tol


def test_reference_unittests_ported(cuda, golden):
    """tests/test_rec/test_reconstruction.py:88-202 of the reference."""
    g = golden("unittest")
    mat, s360 = g["mat"], g["sino_360"]
    s180 = s360[:37]
    ang_deg = g["angles_deg"]
    for fn, key in ((R.fbp_reconstruction, "fbp_180"),
                    (R.bpf_reconstruction, "bpf_180")):
        rec1 = fn(s180.copy(), 32, apply_log=False, gpu=True)
        assert np.max(np.abs(mat - rec1)) <= 0.1
        assert O.rel_l2(rec1, g[key]) < TOL
        rec2 = fn(s360.copy(), 32, angles=np.deg2rad(ang_deg),
                  apply_log=False, gpu=True)
        assert np.max(np.abs(mat - rec2)) <= 0.1
        stack = np.pad(np.expand_dims(s180, 1), ((0, 0), (2, 2), (0, 0)),
                       mode="edge")
        rs = fn(stack.copy(), 32, apply_log=False, gpu=True, ratio=0.0,
                ncore=1)
        assert np.max(np.abs(mat - rs[:, 0, :])) <= 0.1 and rs.shape[1] == 5
        rs = fn(stack.copy(), 32, apply_log=False, gpu=True, ratio=1.0,
                ncore=None)
        assert np.max(np.abs(mat - rs[:, 0, :])) <= 0.1
        rs = fn(stack.copy(), 32, apply_log=False, gpu=False,
                angles=np.deg2rad(ang_deg[:37]), ratio=0.0, ncore=1)
        assert np.median(np.abs(mat - rs[:, 0, :])) <= 0.2
        with pytest.warns(Warning):
            fn(s180.copy(), 32, apply_log=True)
        with pytest.raises(ValueError):
            fn(s180, 32, np.deg2rad(ang_deg), apply_log=False)
        with pytest.raises(ValueError):
            fn(s180, -1, apply_log=False)


def test_torch_inputs_stay_on_device(cuda):
    s, ang, _ = phantom.ellipse_sinogram(2, 90, 128, 63.5)
    t = torch.from_numpy(s).cuda()
    rec = R.fbp_reconstruction(t, 63.5, angles=ang, apply_log=False)
    assert isinstance(rec, torch.Tensor) and rec.is_cuda
    ref = O.fbp_reconstruction(s, 63.5, angles=ang, apply_log=False)
    assert O.rel_l2(rec.cpu().numpy(), ref) < TOL


# ------------------------------------------------ full single-slice sizes
def _fbp_oracle_fast(sino, center, angles, pad=None):
    """FP64 FBP with the C FP64 back-projector (oracle at full size)."""
    nrow, ncol = sino.shape
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    f = O.apply_ramp_filter(sino, None, "hann", pad, "edge")
    rec = cpu_port.back_projection(f.astype(np.float32), angles, center,
                                   ref_arith=False)
    # the FP64 back-projector takes float32 taps; the filter error of that
    # rounding (~6e-8) is far below the tolerance
    mask = O.make_circle_mask(ncol, 1.0)
    return rec * mask * (np.pi / (nrow - 1))


@pytest.mark.parametrize("ncol,nrow,cen", [(1024, 900, 511.5),
                                           (2560, 1801, 1278.3)])
def test_full_size_single_slice(cuda, ncol, nrow, cen):
    """The benchmark shapes: 1024^2 x 900 and one 2560^2 x 1801 slice."""
    s, ang, _ = phantom.ellipse_sinogram(1000 + ncol, nrow, ncol, cen,
                                         photons=1e4)
    got = R.fbp_reconstruction(s, cen, angles=ang, apply_log=False)
    ref = _fbp_oracle_fast(s, cen, ang)
    err = O.rel_l2(got, ref)
    assert err < TOL, err


def test_host_stack_streamed_in_slabs(cuda):
    """A NumPy stack goes through the device slab by slab (copies overlapped
    with compute); the result equals the device-resident path, and `out`
    receives it in place."""
    rng = np.random.default_rng(4)
    nrow, nslice, ncol = 91, 70, 96
    s3 = np.stack([phantom.ellipse_sinogram(700 + k, nrow, ncol, 47.3)[0]
                   for k in range(nslice)], axis=1)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    got = R.fbp_reconstruction(s3, 47.3, angles=ang, apply_log=False)
    assert got.shape == (ncol, nslice, ncol) and got.dtype == np.float32
    dev = R.fbp_reconstruction(torch.from_numpy(s3).cuda(), 47.3, angles=ang,
                               apply_log=False).cpu().numpy()
    assert np.array_equal(got, dev)
    out = np.full((ncol, nslice, ncol), np.nan, np.float32)
    ret = R.fbp_reconstruction(s3, 47.3, angles=ang, apply_log=False, out=out)
    assert ret is out and np.array_equal(out, dev)
    for k in (0, 33, 69):
        ref = O.fbp_reconstruction(s3[:, k], 47.3, angles=ang, apply_log=False)
        assert O.rel_l2(got[:, k], ref) < TOL
    del rng


@pytest.mark.parametrize("ncol,cen", [(33, 16.0), (257, 130.2), (1000, 499.5)])
def test_single_slice_tile_variant_1(cuda, ncol, cen):
    s, ang, _ = phantom.ellipse_sinogram(ncol, 121, ncol, cen)
    t = torch.from_numpy(s).cuda()[:, None]
    ref = O.back_projection(s, ang, cen)
    for v in (0, 1):
        got = R.backproject(t, ang, cen, variant=v)[:, 0].cpu().numpy()
        assert O.rel_l2(got, ref) < 1e-6


@pytest.mark.parametrize("storage,bound", [("float16", 5e-4), ("bfloat16", 4e-3)])
def test_reduced_storage_stack(cuda, storage, bound):
    """Stacks (4- and 2-slice CTAs keep 16-bit pairs in shared memory):
    FP32 accumulation, error bounded by the storage precision."""
    nrow, ncol, nslice = 181, 192, 6
    s3 = np.stack([phantom.ellipse_sinogram(60 + k, nrow, ncol, 95.3)[0]
                   for k in range(nslice)], axis=1)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    t = torch.from_numpy(s3).cuda()
    got = R.fbp_reconstruction(t, 95.3, angles=ang, apply_log=False,
                               storage=storage).cpu().numpy()
    for k in range(nslice):
        ref = O.fbp_reconstruction(s3[:, k], 95.3, angles=ang,
                                   apply_log=False)
        assert O.rel_l2(got[:, k], ref) < bound, (k, O.rel_l2(got[:, k], ref))
