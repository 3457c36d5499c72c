"""Centre search by slice metrics (reconstruction.py:1212-1458).

CPU tests pin the oracle (``oracle/center_oracle.py``) to vectors produced
by the reference itself (``tests/golden/golden_center.npz``) and check the C
ABI's argument errors.  GPU tests hold the device path to:

- the pre-steps (Gaussian smoothing, linear zoom): bit-exact with scipy;
- the metrics of a fixed image: entropy to 1e-12, sharpness to 1e-6
  relative (the reference takes a float32 mean, the device an FP64 sum);
- every candidate's metric: entropy and sharpness of the candidate images
  within 2e-4 relative of the reference's -- a 1e-6 difference between two
  float32 reconstructions moves a few pixels across a histogram-bin edge --
  and the chosen centre among the reference's best within that tolerance.
"""
import warnings

import numpy as np
import pytest

from algotom_b200 import _native as nat
from oracle import center_oracle as C

CASES = {
    "fbp_entropy": dict(metric="entropy", method="fbp", sigma=2, ratio=1.0),
    "fbp_sharp": dict(metric="sharpness", method="fbp", sigma=0, ratio=1.0),
    "fbp_entropy_r0": dict(metric="entropy", method="fbp", sigma=1,
                           ratio=0.0),
    "fbp_entropy_nomask": dict(metric="entropy", method="fbp", sigma=2,
                               ratio=None),
    "bpf_entropy": dict(metric="entropy", method="bpf", sigma=2, ratio=1.0),
    "bpf_sharp": dict(metric="sharpness", method="bpf", sigma=2, ratio=1.0),
}
FINDS = {
    "z1": dict(zoom=1.0),
    "z05": dict(zoom=0.5),
    "z08_default_angles": dict(zoom=0.8, angles=None),
    "sharp": dict(zoom=1.0, metric="sharpness"),
    "bpf": dict(zoom=1.0, method="bpf"),
    "r0": dict(zoom=1.0, radius=0.0),
}
METRIC_RTOL = 2e-4


def _best_within(centers, ref_metrics, chosen, rtol):
    """``chosen`` is a centre whose reference metric is within rtol of the
    reference's minimum."""
    k = int(np.argmin(np.abs(np.asarray(centers) - chosen)))
    assert abs(centers[k] - chosen) < 1e-9
    lo = np.min(ref_metrics)
    return ref_metrics[k] - lo <= rtol * abs(lo)


# ------------------------------------------------------------- oracle (CPU)
@pytest.mark.parametrize("sigma", [1, 2, 3.5])
def test_oracle_gaussian_bit_exact(golden, sigma):
    g = golden("center")
    got = C.gaussian_filter_rows(g["sino"], sigma)
    assert np.array_equal(got, g["gauss__%s" % sigma])


def test_oracle_gaussian_narrow_rows(golden):
    g = golden("center")  # 5 columns, radius 8: repeated reflection
    assert np.array_equal(C.gaussian_filter_rows(g["narrow"], 2),
                          g["gauss__narrow__2"])


@pytest.mark.parametrize("z", [0.5, 0.8, 0.33])
def test_oracle_zoom_bit_exact(golden, z):
    g = golden("center")
    got = C.zoom_linear(g["sino"], z)
    assert np.array_equal(got, g["zoom__%s" % z])


def test_oracle_metrics_of_fixed_image(golden):
    g = golden("center")
    img = g["metric_img"]
    lv = C.normalise_u8(img, img.min(), img.max())
    assert C.histogram_entropy(lv) == pytest.approx(
        float(g["metric__entropy"]), rel=1e-13)
    assert C.edge_sharpness(img) == pytest.approx(
        float(g["metric__sharpness"]), rel=1e-6)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_candidate_metrics(golden, name):
    g = golden("center")
    cen = float(g["center"])
    cs, ms = C.slice_metrics(g["sino"], cen - 3, cen + 3, 0.5,
                             angles=g["angles"], apply_log=False,
                             **CASES[name])
    ref = g["list__%s__metrics" % name]
    assert np.allclose(cs, g["list__%s__centers" % name])
    assert np.max(np.abs(ms - ref) / np.abs(ref)) < METRIC_RTOL
    assert _best_within(cs, ref, cs[np.argmin(ms)], METRIC_RTOL)


def test_oracle_log_input(golden):
    g = golden("center")
    cen = float(g["center"])
    cs, ms = C.slice_metrics(g["trans"], cen - 2, cen + 2, 1.0,
                             angles=g["angles"], apply_log=True)
    ref = g["list__log__metrics"]
    assert np.max(np.abs(ms - ref) / np.abs(ref)) < METRIC_RTOL


def test_oracle_integer_counts(golden):
    """uint16 counts: scipy smooths them into uint16, truncated toward
    zero, and the -log follows in float32."""
    g = golden("center")
    cen = float(g["center"])
    got = C.gaussian_filter_rows(g["counts"], 2)
    assert got.dtype == np.uint16
    assert np.array_equal(got, g["gauss__u16__2"])
    cs, ms = C.slice_metrics(g["counts"], cen - 2, cen + 2, 1.0,
                             angles=g["angles"], apply_log=True, sigma=2)
    ref = g["list__u16__metrics"]
    assert np.array_equal(cs, g["list__u16__centers"])
    assert np.max(np.abs(ms - ref) / np.abs(ref)) < METRIC_RTOL


@pytest.mark.parametrize("name", sorted(FINDS))
def test_oracle_find_center(golden, name):
    g = golden("center")
    cen = float(g["center"])
    kw = dict(FINDS[name])
    kw.setdefault("angles", g["angles"])
    got = C.find_center(g["sino"], cen - 6, cen + 6, step=0.25,
                        apply_log=False, **kw)
    assert abs(got - float(g["find__%s" % name])) < 1e-9


# ------------------------------------------------------------- host + ABI
def test_gaussian_weights_match_oracle():
    from algotom_b200.rec import center as CC
    for s in (0.5, 1, 2, 3.5, 10):
        assert np.array_equal(CC._gaussian_weights(s), C.gaussian_weights(s))


def test_empty_search_range_raises():
    from algotom_b200.rec import reconstruction as R
    with pytest.raises(ValueError, match="Invalid searching parameters"):
        R._find_center_based_slice_metric(np.ones((5, 8), np.float32), 4, 4)


def test_abi_argument_errors():
    lib = nat.load()
    one = 1
    assert lib.atb_gaussian_rows(None, 8, 4, 8, None, 2, None, 8, 0,
                                 None) == -1
    assert lib.atb_gaussian_rows(one, 8, 4, 8, one, 9000, 2, 8, 0,
                                 None) == -3
    assert lib.atb_gaussian_rows(one, 8, 4, 8, one, 2, one, 8, 1,
                                 None) == -1
    assert lib.atb_zoom_linear(one, 8, 0, 8, 2, 8, 4, 4, None) == -1
    assert lib.atb_zoom_linear(one, 8, 4, 8, 2, 8, 70000, 4, None) == -3
    assert lib.atb_image_range(one, 8, 0, 8, one, one, None) == -1
    assert lib.atb_slice_metric_workspace(2, 8, 8, 0) == 2 * 256 * 8
    assert lib.atb_slice_metric_workspace(2, 8, 8, 7) == 0
    assert lib.atb_slice_metric(one, 64, 8, 2, 8, 8, 0, 0.0, 1.0, one, 16,
                                one, None) == -1  # workspace too small
    assert lib.atb_slice_metric(one, 64, 8, 2, 8, 8, 5, 0.0, 1.0, one,
                                1 << 20, one, None) == -1  # unknown metric
    assert b"metric" in nat.load().atb_last_error()


# ------------------------------------------------------------- device (GPU)
def _dev(x):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x), device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("sigma", [1, 2, 3.5])
def test_gaussian_rows_bit_exact(cuda, golden, sigma):
    from algotom_b200.rec import center as CC
    g = golden("center")
    got = CC.gaussian_filter_rows(_dev(g["sino"]), sigma).cpu().numpy()
    assert np.array_equal(got, g["gauss__%s" % sigma])
    got = CC.gaussian_filter_rows(_dev(g["narrow"]), 2).cpu().numpy()
    assert np.array_equal(got, g["gauss__narrow__2"])


@pytest.mark.gpu
def test_gaussian_rows_integer_counts(cuda, golden):
    """to_int: each result truncated toward zero, as scipy's uint16."""
    from algotom_b200.rec import center as CC
    g = golden("center")
    x = _dev(g["counts"].astype(np.float32))
    got = CC.gaussian_filter_rows(x, 2, to_int=True).cpu().numpy()
    assert np.array_equal(got, g["gauss__u16__2"].astype(np.float32))
    rng = np.random.default_rng(3)
    for dt, lo, hi in ((np.uint16, 0, 65536), (np.int16, -3000, 3000)):
        v = rng.integers(lo, hi, (9, 300)).astype(dt)
        for sigma in (0.7, 3, 5):  # register windows and shared-memory taps
            got = CC.gaussian_filter_rows(_dev(v.astype(np.float32)), sigma,
                                          to_int=True).cpu().numpy()
            assert np.array_equal(got, C.gaussian_filter_rows(v, sigma)
                                  .astype(np.float32)), (dt, sigma)


@pytest.mark.gpu
def test_integer_sinogram_search_matches_reference(cuda, golden):
    from algotom_b200.rec import reconstruction as R
    g = golden("center")
    cen = float(g["center"])
    counts = g["counts"].copy()
    cs, ms = R._find_center_based_slice_metric(
        counts, cen - 2, cen + 2, 1.0, angles=g["angles"], sigma=2,
        apply_log=True, return_metric=True)
    ref = g["list__u16__metrics"]
    assert np.array_equal(cs, g["list__u16__centers"])
    assert np.max(np.abs(ms - ref) / np.abs(ref)) < METRIC_RTOL
    assert np.array_equal(counts, g["counts"])


def test_integer_input_detection():
    """Which inputs scipy's filters would store as integers."""
    import torch
    from algotom_b200.rec.center import _integer_input
    assert _integer_input(np.zeros(3, np.uint16))
    assert _integer_input(np.zeros(3, np.int32))
    assert _integer_input([1, 2, 3])
    assert not _integer_input(np.zeros(3, np.float32))
    assert not _integer_input([1.0, 2.0])
    assert _integer_input(torch.zeros(3, dtype=torch.int16))
    assert not _integer_input(torch.zeros(3))
    assert not _integer_input(torch.zeros(3, dtype=torch.bool))
    assert not _integer_input(torch.zeros(3, dtype=torch.complex64))


def test_centre_groups():
    from algotom_b200.rec.center import _centre_groups
    g = _centre_groups(np.arange(1270.3, 1278.3, 0.25))
    assert len(g) == 4 and all(x[3] == 1 and x[4] == 8 for x in g)
    assert [x[0] for x in g] == [0, 1, 2, 3]
    assert _centre_groups(np.arange(40.0, 50.0, 1.0)) == [(0, 1, 40.0, 1, 10)]
    g = _centre_groups(np.arange(40.0, 50.0, 0.3))  # 10 classes, 3 px apart
    assert len(g) == 10 and all(x[3] == 3 for x in g)
    for r, ncls, c0, sp, cnt in g:
        c = np.float32(np.arange(40.0, 50.0, 0.3)[r::ncls])
        assert np.array_equal(c.astype(np.float64), c0 + sp * np.arange(cnt))
    assert _centre_groups([5.0]) is None
    assert _centre_groups(np.linspace(10.0, 11.0, 40) ** 1.5) is None


@pytest.mark.gpu
@pytest.mark.parametrize("ncol,nrow,c0,spacing,count,edge_pad,r2", [
    (256, 181, 127.3, 1, 11, 0, 128.0 ** 2),   # 4 + 4 + 2 + 1 centres
    (200, 91, 3.25, 2, 9, 0, -1.0),            # near the first edge, no mask
    (200, 91, 160.5, 3, 13, 0, -1.0),          # last centres near ncol - 1
    (256, 120, 100.75, 1, 8, 1, -1.0),         # BPF: edge padding
    (96, 60, 10.0, 7, 12, 0, 48.0 ** 2)])
def test_centre_group_equals_single_centres(cuda, ncol, nrow, c0, spacing,
                                            count, edge_pad, r2):
    """atb_backproject_centers image m equals the single-centre
    back-projection at c0 + m * spacing (only the FP32 partial sums are
    grouped differently), with TMA and cp.async staging identical."""
    import torch
    from algotom_b200 import _native as nat
    from algotom_b200.rec import reconstruction as R
    rng = np.random.default_rng(ncol + count)
    s = rng.standard_normal((nrow, ncol)).astype(np.float32)
    ang = np.concatenate([[0.0, np.pi / 2, np.pi / 4], rng.uniform(0, np.pi,
                                                                   nrow)])
    ang = ang[:nrow]
    t = torch.from_numpy(s).to(cuda)
    trig = R._trig(ang, t.device)
    outs = []
    for flags in (0, 16):
        out = torch.full((count, ncol, ncol), np.nan, device=cuda)
        nat.call("atb_backproject_centers", t.data_ptr(), t.stride(0), nrow,
                 ncol, trig.data_ptr(), float(np.float32(c0)), spacing,
                 count, edge_pad, r2, 0.5, out.data_ptr(), out.stride(1),
                 out.stride(0), flags, R._stream_ptr(t.device))
        outs.append(out)
    assert torch.equal(outs[0], outs[1])
    assert nat.call("atb_backproject_status", 0) == 0
    for m in range(count):
        c = float(np.float32(c0)) + m * spacing
        one = R.backproject(t[:, None], ang, c, edge_pad=bool(edge_pad),
                            mask_r2=r2, scale=0.5, trig=trig)[:, 0]
        got = outs[0][m]
        err = (got - one).abs().max().item()
        assert err <= 1e-5 * one.abs().max().item(), (m, c, err)


def test_centre_group_launch_plan(monkeypatch):
    """The host's calls for a search at step 0.25: one
    atb_backproject_centers per residue class, each writing every fourth
    image (first image r, image stride 4 images) at float32 centres 1 px
    apart; ratio=0.0 (a mask per centre) falls back to the batch path."""
    import torch
    from algotom_b200.rec import center as CC
    from algotom_b200.rec import reconstruction as R
    calls = []
    monkeypatch.setattr(CC.nat, "call", lambda name, *a: calls.append(
        (name, a)) or 1)
    monkeypatch.setattr(R, "_stream_ptr", lambda dev=None: 0)
    monkeypatch.setattr(CC, "_backproject_items",
                        lambda items, dev, v: calls.append(
                            ("batch", len(items))))
    ncol, nrow = 64, 30
    src = CC._Source.__new__(CC._Source)
    src.method, src.nrow, src.ncol = "fbp", nrow, ncol
    src.sino = torch.zeros((nrow, ncol))
    src.angles = np.linspace(0.0, np.pi, nrow)
    src.src, src.src_rs = torch.zeros((nrow, 1, ncol)), ncol
    src.trig = torch.zeros((nrow, 2), dtype=torch.float64)
    cs = np.arange(30.3, 32.3, 0.25)   # 8 candidates, 4 classes of 2
    out = src.reconstruct(cs, 1.0)
    assert out.shape == (8, ncol, ncol)
    assert [c[0] for c in calls] == ["atb_backproject_centers"] * 4
    esize = out.element_size()
    for r, (_, a) in enumerate(calls):
        assert a[5] == float(np.float32(cs[r]))       # first centre
        assert a[6] == 1 and a[7] == 2                  # spacing, count
        assert a[8] == 0 and a[10] == R._scale(nrow)    # FBP: no edge pad
        assert (a[11] - out.data_ptr()) == r * ncol * ncol * esize
        assert a[12] == ncol and a[13] == 4 * ncol * ncol
    calls.clear()
    src.reconstruct(cs, 0.0)                            # mask per centre
    assert calls == [("batch", 8)]


def test_centre_group_argument_errors():
    """Rejected before any device work (the pointers are never read)."""
    lib = nat.load()
    args = (16, 64, 4, 64, 16)
    tail = (0, -1.0, 1.0, 16, 64, 4096, 0, None)
    assert lib.atb_backproject_centers(*args, 10.0, 57, 2, *tail) == -3
    assert lib.atb_backproject_centers(*args, 10.0, 0, 2, *tail) == -3
    assert lib.atb_backproject_centers(*args, 60.0, 2, 3, *tail) == -1
    assert lib.atb_backproject_centers(*args, 10.0, 1, 0, *tail) == -1


@pytest.mark.gpu
@pytest.mark.parametrize("z", [0.5, 0.8, 0.33])
def test_zoom_bit_exact(cuda, golden, z):
    from algotom_b200.rec import center as CC
    g = golden("center")
    got = CC.zoom_image(_dev(g["sino"]), z).cpu().numpy()
    assert np.array_equal(got, g["zoom__%s" % z])


@pytest.mark.gpu
def test_image_range_and_fixed_image_metrics(cuda, golden):
    import torch
    from algotom_b200.rec import center as CC
    g = golden("center")
    img = g["metric_img"]
    lo, hi = CC.image_range(_dev(img))
    assert lo == img.min() and hi == img.max()
    stack = _dev(np.stack([img, img[::-1].copy(), 2 * img]))
    e = CC.slice_metrics(stack, "entropy", lo, hi)
    levels = [C.normalise_u8(x, lo, hi) for x in stack.cpu().numpy()]
    ref = [C.histogram_entropy(lv) for lv in levels]
    assert e[0] == pytest.approx(float(g["metric__entropy"]), rel=1e-12)
    assert np.allclose(e, ref, rtol=1e-12, atol=0)
    s = CC.slice_metrics(stack, "sharpness")
    assert s[0] == pytest.approx(float(g["metric__sharpness"]), rel=1e-6)
    assert np.allclose(s, [C.edge_sharpness(x) for x in
                           stack.cpu().numpy()], rtol=1e-12, atol=0)
    nan = img.copy()
    nan[3, 4] = np.nan
    lo, hi = CC.image_range(_dev(nan))
    assert np.isnan(lo) and np.isnan(hi)
    # non-contiguous batch (every other image of a view)
    s2 = CC.slice_metrics(torch.cat([stack, stack])[::2], "sharpness")
    assert np.array_equal(s2, CC.slice_metrics(torch.cat([stack, stack])
                                               [::2].contiguous(),
                                               "sharpness"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_candidate_metrics_match_reference(cuda, golden, name):
    from algotom_b200.rec import reconstruction as R
    g = golden("center")
    cen = float(g["center"])
    cs, ms = R._find_center_based_slice_metric(
        g["sino"].copy(), cen - 3, cen + 3, 0.5, angles=g["angles"],
        apply_log=False, return_metric=True, **CASES[name])
    ref = g["list__%s__metrics" % name]
    assert np.allclose(cs, g["list__%s__centers" % name])
    assert ms.dtype == np.float64
    assert np.max(np.abs(ms - ref) / np.abs(ref)) < METRIC_RTOL
    best = R._find_center_based_slice_metric(
        g["sino"].copy(), cen - 3, cen + 3, 0.5, angles=g["angles"],
        apply_log=False, return_metric=False, **CASES[name])
    assert best == cs[np.argmin(ms)]
    assert _best_within(cs, ref, best, METRIC_RTOL)


@pytest.mark.gpu
def test_candidate_images_equal_single_reconstructions(cuda, golden):
    """The batched candidates equal fbp/bpf_reconstruction one by one."""
    from algotom_b200.rec import center as CC
    from algotom_b200.rec import reconstruction as R
    g = golden("center")
    sino, ang = g["sino"], g["angles"]
    cs = [44.0, 46.3, 47.75]
    for method, fn in (("fbp", R.fbp_reconstruction),
                       ("bpf", R.bpf_reconstruction)):
        for ratio in (1.0, 0.0, None):
            imgs = CC.reconstruct_centers(_dev(sino), cs, ang, method,
                                          ratio).cpu().numpy()
            for k, c in enumerate(cs):
                one = fn(sino.copy(), c, angles=ang, ratio=ratio,
                         apply_log=False)
                assert np.allclose(imgs[k], one, rtol=0, atol=1e-6 * max(
                    1.0, float(np.abs(one).max()))), (method, ratio, c)


@pytest.mark.gpu
def test_log_input_warns_and_matches(cuda, golden):
    from algotom_b200.rec import reconstruction as R
    g = golden("center")
    cen = float(g["center"])
    t = g["trans"].copy()
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        cs, ms = R._find_center_based_slice_metric(
            t, cen - 2, cen + 2, 1.0, angles=g["angles"], apply_log=True)
    # sigma = 2 smooths the single zero away before the check, so the
    # reference does not warn either; the caller's array is left alone
    assert not any("logarithm" in str(w.message) for w in caught)
    ref = g["list__log__metrics"]
    assert np.max(np.abs(ms - ref) / np.abs(ref)) < METRIC_RTOL
    assert np.array_equal(t, g["trans"])


@pytest.mark.gpu
def test_sigma0_log_mutates_callers_array(cuda, golden):
    """With no smoothing the reference repairs values <= 0 in the array it
    was given (reconstruction.py:1319-1325)."""
    from algotom_b200.rec import reconstruction as R
    g = golden("center")
    cen = float(g["center"])
    t = g["trans"].copy()
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        R._find_center_based_slice_metric(t, cen - 1, cen + 1, 1.0,
                                          angles=g["angles"], sigma=0)
    assert any("logarithm" in str(w.message) for w in caught)
    assert t[7, 11] == np.float32(1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FINDS))
def test_find_center_matches_reference(cuda, golden, name):
    from algotom_b200.rec import reconstruction as R
    g = golden("center")
    cen = float(g["center"])
    kw = dict(FINDS[name])
    kw.setdefault("angles", g["angles"])
    got = R.find_center_based_slice_metric(g["sino"].copy(), cen - 6,
                                           cen + 6, step=0.25,
                                           apply_log=False, **kw)
    # the fine pass's metric of the chosen centre is the reference's best
    # (or within the metric tolerance of it)
    ref = float(g["find__%s" % name])
    if abs(got - ref) > 1e-9:
        kw.pop("zoom", None)
        radius = kw.pop("radius", 2)
        assert radius != 0.0, "coarse passes must agree exactly"
        cs = np.arange(ref - 3, ref + 3.25, 0.25)
        _, ms = R._find_center_based_slice_metric(
            g["sino"].copy(), cs[0], cs[-1] + 0.1, 0.25, apply_log=False,
            **{k: v for k, v in kw.items()})
        k_got = int(np.argmin(np.abs(cs - got)))
        k_ref = int(np.argmin(np.abs(cs - ref)))
        assert ms[k_got] - ms[k_ref] <= METRIC_RTOL * abs(ms[k_ref])


@pytest.mark.gpu
def test_reference_unittest_case(cuda, golden):
    """Port of test_reconstruction.py:242-272 with the FBP method."""
    from algotom_b200.rec import reconstruction as R
    g = golden("unittest")
    sino_180 = g["sino_360"][:37]
    center = 32
    got = R.find_center_based_slice_metric(
        sino_180.copy(), center - 2, center + 2, step=0.25, radius=2,
        zoom=1.0, method="fbp", gpu=True, angles=None, ratio=1.0,
        filter_name="hann", apply_log=False, ncore=None, sigma=1,
        metric_function=None)
    assert abs(got - center) < 0.1

    def get_negative(mat, n=2):
        return np.abs(np.mean(mat[mat < 0.0])) ** n

    got = R.find_center_based_slice_metric(
        sino_180.copy(), center - 2, center + 2, step=0.25, radius=2,
        zoom=1.0, method="fbp", angles=None, ratio=1.0, filter_name="hann",
        apply_log=False, sigma=1, metric_function=get_negative, n=2)
    cs, ms = R._find_center_based_slice_metric(
        sino_180.copy(), got - 1, got + 1.1, 0.25, angles=None,
        apply_log=False, sigma=1, metric_function=get_negative, n=2)
    assert got in cs and ms[list(cs).index(got)] == np.min(ms)
    inv = R._find_center_based_slice_metric(
        sino_180.copy(), got - 1, got + 1.1, 0.25, apply_log=False, sigma=1,
        metric_function=get_negative, invert_metric=True, n=2)
    assert np.allclose(inv[1], np.max(ms) - ms)


@pytest.mark.gpu
def test_errors(cuda):
    from algotom_b200.rec import reconstruction as R
    with pytest.raises(ValueError, match="Empty image"):
        R._find_center_based_slice_metric(np.zeros((10, 16), np.float32),
                                          7, 9, 1, apply_log=False)
    with pytest.raises(ValueError, match="Center is out of the range"):
        R._find_center_based_slice_metric(
            np.random.default_rng(0).random((10, 16)).astype(np.float32),
            14, 18, 1, apply_log=False, metric="sharpness")
    with pytest.raises(NotImplementedError):
        R._find_center_based_slice_metric(np.ones((10, 16), np.float32),
                                          7, 9, 1, apply_log=False,
                                          method="gridrec")
