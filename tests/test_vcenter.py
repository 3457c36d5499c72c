"""Centre search on a vertical slice (find_center_vertical_slice,
algotom/rec/vertrec.py:1264-1383).

CPU tests pin the oracle (``oracle/vertical_oracle.py``) to vectors made by
the reference's CPU path (``tests/golden/golden_vcenter.npz``): the
projection smoothing bit-exactly, the metrics of every candidate centre to
the tolerances below, the best centre exactly.  GPU tests hold the device
path -- column and row Gaussian kernels, one vertical back-projection of all
candidates with a centre per line, device metrics -- to the same vectors.

Tolerances: the slices agree with the reference to ~1e-6 relative, so
sharpness and autocorrelation agree to 1e-5 relative; the entropy counts
pixels in 256 levels, and a pixel within 1e-6 of a level boundary may land
on the other side (one pixel moves the entropy by ~0.3 of ~3e4), so it is
held to 1e-4 of the metric's scale.
"""
import warnings

import numpy as np
import pytest

from algotom_b200 import _native as nat
from oracle import vertical_oracle as V

SIGMAS = (3, 1.5, 0.7)
CASES = {
    "entropy": dict(),
    "sharpness": dict(metric="sharpness"),
    "autocorr": dict(metric="autocorrelation"),
    "entropy_before": dict(ramp_filter="before", sigma=1.5),
    "sharp_nomask": dict(metric="sharpness", masking=False, sigma=0,
                         alpha=30.0, slice_index=20),
    "entropy_invert": dict(invert_metric=True, chunk_size=16, sigma=0.7),
    "autocorr_angles": dict(metric="autocorrelation", alpha=60.0,
                            slice_index=40, angles=True, chunk_size=None),
}
ENTROPY_SCALE = 3.0e4  # |entropy| of these slices


def _kwargs(g, name):
    kw = dict(CASES[name])
    idx = kw.pop("slice_index", 32)
    if kw.get("angles") is True:
        kw["angles"] = g["angles"]
    return idx, kw


def _check(name, got, ref):
    if "entropy" in name:
        # uint16 counts: the reference sums -log(counts) ~ -10.6 per sample
        # in float32, so its slices are 2e-6 (not 1e-6) from the FP64 ones
        # and twice as many pixels sit near a level boundary
        tol = 3e-4 if name.startswith("u16") else 1e-4
        err = np.max(np.abs(np.asarray(got, np.float64) - ref))
        assert err <= tol * ENTROPY_SCALE, (name, err)
    else:
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err < 1e-5, (name, err)
    assert np.argmin(got) == np.argmin(ref), name


# ------------------------------------------------------------- CPU
@pytest.mark.parametrize("sigma", SIGMAS)
def test_oracle_smoothing_bit_exact(golden, sigma):
    g = golden("vcenter")
    assert np.array_equal(V.smooth_projections(g["trans"], sigma),
                          g["smooth__%s" % sigma])
    assert np.array_equal(V.smooth_projections(g["tall"], sigma),
                          g["smooth_tall__%s" % sigma])


U16_CASES = {
    "u16_entropy": dict(),
    "u16_sharp_before_nolog": dict(metric="sharpness", apply_log=False,
                                   sigma=1.5, ramp_filter="before"),
}


@pytest.mark.parametrize("sigma", (3, 1.5))
def test_oracle_smoothing_integer_counts(golden, sigma):
    """uint16 projections: each pass truncated toward zero, as scipy's."""
    g = golden("vcenter")
    got = V.smooth_projections(g["counts"], sigma)
    assert got.dtype == np.uint16
    assert np.array_equal(got, g["smooth_u16__%s" % sigma])


@pytest.mark.parametrize("name", sorted(U16_CASES))
def test_oracle_search_integer_counts(golden, name):
    g = golden("vcenter")
    cs, ms = V.find_center_vertical_slice(g["counts"], 32, 28.0, 35.0,
                                          step=0.5, **U16_CASES[name])
    assert np.array_equal(cs, g["vc__%s__centers" % name])
    _check(name, ms, g["vc__%s__metrics" % name])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_search(golden, name):
    g = golden("vcenter")
    idx, kw = _kwargs(g, name)
    cs, ms = V.find_center_vertical_slice(g["trans"], idx, 28.0, 35.0,
                                          step=0.5, **kw)
    assert np.array_equal(cs, g["vc__%s__centers" % name])
    _check(name, ms, g["vc__%s__metrics" % name])


def _get_negative(mat, n=2):
    return np.abs(np.mean(mat[mat < 0.0])) ** n


CUBE = ("autocorrelation", "entropy", "sharpness", "custom")


def _cube_kwargs(metric):
    kw = dict(step=1.0, invert_metric=True)
    if metric == "custom":
        kw.update(metric_function=_get_negative, n=2)
    else:
        kw.update(metric=metric, masking=False)
    return kw


@pytest.mark.parametrize("metric", CUBE)
def test_oracle_cube_phantom(golden, metric):
    """The reference's own search test (tests/test_rec/test_vertrec.py:
    498-539): the best centre is the phantom's, 30."""
    g = golden("vcenter")
    cs, ms = V.find_center_vertical_slice(g["cube_projs"], 30, 25, 39,
                                          **_cube_kwargs(metric))
    assert np.array_equal(cs, g["cube__%s__centers" % metric])
    _check("entropy" if metric == "entropy" else metric, ms,
           g["cube__%s__metrics" % metric])
    assert abs(cs[np.argmin(ms)] - 30) < 0.5


def test_abi_argument_errors():
    lib = nat.load()
    one = 1
    assert lib.atb_gaussian_cols(None, 64, 8, 1, 8, 8, one, 2, one, 64, 8,
                                 0, None) == -1
    assert lib.atb_gaussian_cols(one, 64, 8, 1, 8, 8, one, 2, one, 64, 8,
                                 0, None) == -1  # in place
    assert lib.atb_gaussian_cols(one, 64, 8, 1, 8, 8, one, 701, 2, 64, 8,
                                 1, None) == -3
    assert lib.atb_gaussian_cols(one, 64, 8, 0, 8, 8, one, 2, 2, 64, 8,
                                 0, None) == -1
    assert lib.atb_slice_entropy64(one, 64, 8, 1, 8, 8, 0.0, 1.0, one, 16,
                                   one, None) == -1  # workspace too small
    assert lib.atb_slice_entropy64(None, 64, 8, 1, 8, 8, 0.0, 1.0, one,
                                   4096, one, None) == -1
    assert b"atb_slice_entropy64" in lib.atb_last_error()


def test_gaussian_slab_passes_truncation_flag(monkeypatch):
    """Both passes get to_int (the argument before the stream)."""
    import torch
    from algotom_b200.rec import vertrec as VR
    calls = []
    monkeypatch.setattr(VR.nat, "call", lambda name, *a: calls.append(
        (name, a)))
    monkeypatch.setattr(VR.R, "_stream_ptr", lambda dev=None: 0)
    x = torch.zeros((2, 5, 7))
    w = torch.zeros(4, dtype=torch.float64)
    for flag in (False, True):
        calls.clear()
        VR._gaussian_slab(x, w, torch.empty_like(x), torch.empty_like(x),
                          to_int=flag)
        assert [c[0] for c in calls] == ["atb_gaussian_cols",
                                         "atb_gaussian_rows"]
        assert all(c[1][-2] == int(flag) for c in calls)
        assert calls[0][1][3:6] == (2, 5, 7) and calls[0][1][7] == 3


def test_metric_argument_error():
    from algotom_b200.rec import vertrec as VR
    with pytest.raises(ValueError, match="Please select one of three"):
        VR.find_center_vertical_slice(np.ones((4, 3, 8), np.float32), 2,
                                      3.0, 4.0, metric="variance")


# ------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("sigma", SIGMAS)
def test_device_smoothing_bit_exact(cuda, golden, sigma):
    import torch
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    for key, x in (("smooth", g["trans"]), ("smooth_tall", g["tall"])):
        t = torch.as_tensor(x, device=cuda)
        w = torch.from_numpy(VR._gaussian_weights(sigma)).to(cuda)
        tmp, out = torch.empty_like(t), torch.empty_like(t)
        VR._gaussian_slab(t, w, tmp, out)
        assert np.array_equal(out.cpu().numpy(), g["%s__%s" % (key, sigma)])


@pytest.mark.gpu
@pytest.mark.parametrize("sigma", (0.7, 2, 3, 4, 5))
def test_device_smoothing_tiles_and_radii(cuda, sigma):
    """Both forms of each Gaussian pass (register windows up to radius 16,
    shared-memory taps beyond) over several tiles, against the oracle,
    which is bit-exact with scipy."""
    import torch
    from algotom_b200.rec import vertrec as VR
    x = np.random.default_rng(5).random((3, 150, 203)).astype(np.float32)
    t = torch.as_tensor(x, device=cuda)
    w = torch.from_numpy(VR._gaussian_weights(sigma)).to(cuda)
    tmp, out = torch.empty_like(t), torch.empty_like(t)
    VR._gaussian_slab(t, w, tmp, out)
    assert np.array_equal(out.cpu().numpy(), V.smooth_projections(x, sigma))


@pytest.mark.gpu
@pytest.mark.parametrize("sigma", (3, 1.5))
def test_device_smoothing_integer_counts(cuda, golden, sigma):
    import torch
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    t = torch.as_tensor(g["counts"].astype(np.float32), device=cuda)
    w = torch.from_numpy(VR._gaussian_weights(sigma)).to(cuda)
    tmp, out = torch.empty_like(t), torch.empty_like(t)
    VR._gaussian_slab(t, w, tmp, out, to_int=True)
    assert np.array_equal(out.cpu().numpy(),
                          g["smooth_u16__%s" % sigma].astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(U16_CASES))
@pytest.mark.parametrize("where", ("host", "device"))
def test_search_integer_counts_match_reference(cuda, golden, name, where):
    """uint16 projections, from host memory or already on the device."""
    import torch
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    counts = g["counts"].copy()
    projs = counts if where == "host" else torch.as_tensor(counts,
                                                           device=cuda)
    cs, ms = VR.find_center_vertical_slice(
        projs, 32, 28.0, 35.0, step=0.5, gpu=False, show_progress=False,
        return_metric=True, **U16_CASES[name])
    assert np.array_equal(cs, g["vc__%s__centers" % name])
    _check(name, ms, g["vc__%s__metrics" % name])
    assert np.array_equal(counts, g["counts"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_search_matches_reference(cuda, golden, name):
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    idx, kw = _kwargs(g, name)
    trans = g["trans"].copy()
    cs, ms = VR.find_center_vertical_slice(
        trans, idx, 28.0, 35.0, step=0.5, gpu=False, show_progress=False,
        return_metric=True, **kw)
    assert np.array_equal(cs, g["vc__%s__centers" % name])
    assert ms.dtype == np.float64
    _check(name, ms, g["vc__%s__metrics" % name])
    assert np.array_equal(trans, g["trans"])  # the input is not modified


@pytest.mark.gpu
@pytest.mark.parametrize("metric", CUBE)
def test_cube_phantom(cuda, golden, metric):
    """The reference's own search test on the device, CPU-path (gpu=False)
    and GPU-path (gpu=True) positions: the best centre is 30."""
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    projs = g["cube_projs"]
    cs, ms = VR.find_center_vertical_slice(
        projs, 30, 25, 39, gpu=False, show_progress=False,
        return_metric=True, **_cube_kwargs(metric))
    assert np.array_equal(cs, g["cube__%s__centers" % metric])
    _check("entropy" if metric == "entropy" else metric, ms,
           g["cube__%s__metrics" % metric])
    best = VR.find_center_vertical_slice(projs, 30, 25, 39,
                                         show_progress=False,
                                         **_cube_kwargs(metric))
    assert abs(best - 30) < 0.5


@pytest.mark.gpu
def test_search_best_centre_int_range_and_passes(cuda, golden, monkeypatch):
    import torch
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    trans = g["trans"]
    best = VR.find_center_vertical_slice(trans, 32, 28.0, 35.0, step=0.5,
                                         gpu=False, show_progress=False)
    assert best == float(g["vc_best"])
    # integer centres keep NumPy's integer metric array
    cs, ms = VR.find_center_vertical_slice(
        trans, 32, 28, 35, step=1, metric="sharpness", gpu=False,
        show_progress=False, return_metric=True)
    assert ms.dtype == g["vc_int_metrics"].dtype
    assert np.array_equal(cs, g["vc_int_centers"])
    assert np.array_equal(ms, g["vc_int_metrics"])
    # CUDA input, and the candidates split over several passes
    ref = g["vc__entropy__metrics"]
    monkeypatch.setattr(VR, "_SEARCH_BYTES", 8 * 10 * 64 * 4)
    _, ms = VR.find_center_vertical_slice(
        torch.as_tensor(trans, device=cuda), 32, 28.0, 35.0, step=0.5,
        gpu=False, show_progress=False, return_metric=True)
    _check("entropy", ms, ref)


@pytest.mark.gpu
def test_search_gpu_rounding_and_custom_metric(cuda, golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    trans = g["trans"]
    # gpu=True: float32-rounded angles, points and centres
    _, ms = VR.find_center_vertical_slice(
        trans, 32, 28.0, 35.0, step=0.5, metric="sharpness",
        show_progress=False, return_metric=True)
    _check("sharpness", ms, g["vc__sharpness__metrics"])
    seen = []

    def metric_function(recon, scale=1.0):
        seen.append((type(recon), recon.dtype, recon.shape))
        return scale * float(np.abs(recon).sum())
    cs, ms = VR.find_center_vertical_slice(
        trans, 32, 29.0, 31.0, step=1.0, metric=None,
        metric_function=metric_function, scale=2.0, show_progress=False,
        return_metric=True, gpu=False)
    assert seen == [(np.ndarray, np.float64, (10, 64))] * 3
    ver = [VR.vertical_reconstruction(V.smooth_projections(trans, 3), 32, c,
                                      apply_log=True, gpu=False,
                                      show_progress=False,
                                      pad=min(int(0.15 * 64), 150))
           for c in cs]
    rad = int(min(29.0, 64 - 29.0))
    mask = np.zeros(64)
    mask[(64 - 2 * rad) // 2:(64 - 2 * rad) // 2 + 2 * rad] = 1.0
    want = [2.0 * np.abs(v * mask).sum() for v in ver]
    assert np.allclose(ms, want, rtol=1e-6)


@pytest.mark.gpu
def test_search_log_warning_and_repair(cuda, golden):
    from algotom_b200.rec import vertrec as VR
    g = golden("vcenter")
    bad = g["trans"].copy()
    bad[5, 3, 7] = 0.0
    bad[40, 8, 20] = -1.0
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        _, ms = VR.find_center_vertical_slice(
            bad, 32, 29.0, 34.0, step=1.0, sigma=0, metric="sharpness",
            gpu=False, show_progress=False, return_metric=True)
    texts = [str(w.message) for w in caught if "logarithm" in str(w.message)]
    assert texts == list(g["vc_log_warnings"])
    assert np.array_equal(bad, g["vc_log_mutated"])
    _check("sharpness", ms, g["vc_log_metrics"])


@pytest.mark.gpu
@pytest.mark.parametrize("cols", [2560, 75, 61, 71, 1, 2, 3])
def test_autocorrelation_matches_numpy(cuda, cols):
    """The autocorrelation metric (atb_autocorr_rowmax + the row mean)
    against vertrec.py:1255-1261 in FP64 at a 13-smooth even width (2560:
    real transform of half length), a 13-smooth odd one (75: complex
    transform), and widths embedded in 7-smooth lengths of at least
    2 cols - 1 and folded (61 -> 125, odd; 71 -> 144, even), and the
    smallest widths (plans of zero or one stage)."""
    import torch
    from algotom_b200.rec import vertrec as VR
    rng = np.random.default_rng(cols)
    imgs = rng.standard_normal((3, 5, cols)).astype(np.float32)
    imgs[1] += 4.0  # a large mean: the maximum at lag 0
    got = VR._autocorrelation(torch.as_tensor(imgs, device=cuda))
    ref = np.array([V.autocorrelation(im) for im in imgs])
    assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-12
