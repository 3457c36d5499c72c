"""Generate golden input/output vectors by running the reference itself.

Run where the algotom 1.6.0 source tree is available, with
``$ALGOTOM_REF`` naming its root (the directory that holds ``algotom/``),
plus numpy/scipy/numba/joblib:

    ALGOTOM_REF=/path/to/algotom python tests/golden/make_golden.py

The reference imports ``pywt`` and ``h5py`` at module level
(``algotom/util/utility.py:58``, ``algotom/io/loadersaver.py:44``); neither is
used on the FBP/BPF path, so empty stand-in modules are registered first.
``NUMBA_NUM_THREADS=1`` is forced because the reference's multi-threaded
``back_projection_cpu`` races on its output (``prange`` over angles with a
shared ``+=``, ``algotom/rec/reconstruction.py:333,351``); single-threaded it
is deterministic.

Outputs (``tests/golden/*.npz``) hold the inputs next to the reference's
outputs so that tests need neither the reference nor this script.
"""
import os
import sys
import types
import warnings

os.environ["NUMBA_NUM_THREADS"] = "1"
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("ALGOTOM_REF")
if not REF or not os.path.isdir(os.path.join(REF, "algotom")):
    sys.exit("make_golden.py: set ALGOTOM_REF to the root of the algotom "
             "1.6.0 source tree (the directory that holds algotom/); got %r"
             % (REF,))

for _m in ("pywt", "h5py"):
    sys.modules.setdefault(_m, types.ModuleType(_m))
sys.path.insert(0, REF)
sys.path.insert(0, REPO)

import scipy.ndimage as ndi  # noqa: E402
import scipy.signal as ssig  # noqa: E402
import algotom.rec.reconstruction as rec  # noqa: E402
import algotom.util.utility as util  # noqa: E402
from algotom_b200 import phantom  # noqa: E402

WINDOWS = ["hann", "bartlett", "blackman", "hamming", "nuttall", "parzen",
           "triang", None]
PAD_MODES = ["edge", "constant", "reflect", "symmetric", "wrap",
             "linear_ramp", "mean", "maximum", "minimum", "median"]


def _key(*parts):
    return "__".join(str(p) for p in parts)


def make_windows():
    out = {}
    for w in (64, 65):
        for name in WINDOWS:
            out[_key("smooth", name, w)] = rec.make_smoothing_window(name, w)
            out[_key("ramp2d", name, w)] = rec.make_2d_ramp_window(2, w, name)
        for name in ("hann", None):
            out[_key("circ", name, w)] = rec.make_circular_ramp_window(w, name)
    for w, ratio in ((65, 1.0), (64, 0.7), (97, 0.93)):
        out[_key("mask", w, ratio)] = util.make_circle_mask(w, ratio)
    np.savez_compressed(os.path.join(HERE, "golden_windows.npz"), **out)


def make_filter():
    sino, _, _ = phantom.ellipse_sinogram(11, 32, 96, 47.5, photons=1e4)
    out = {"sino": sino}
    for mode in PAD_MODES:
        out[_key("filt", mode, "hann", "None")] = rec.apply_ramp_filter(
            sino, None, "hann", None, mode)
    for name in WINDOWS:
        out[_key("filt", "edge", name, "None")] = rec.apply_ramp_filter(
            sino, None, name, None, "edge")
    for pad in (0, 7, 200):
        for mode in ("edge", "reflect", "wrap"):
            out[_key("filt", mode, "hann", pad)] = rec.apply_ramp_filter(
                sino, None, "hann", pad, mode)
    # odd width: N = ncol + 2 pad odd, H Hermitian
    sino_odd, _, _ = phantom.ellipse_sinogram(12, 24, 81, 40.0, photons=1e4)
    out["sino_odd"] = sino_odd
    out[_key("filtodd", "edge", "hann", "None")] = rec.apply_ramp_filter(
        sino_odd, None, "hann", None, "edge")
    # the reference returns float64; float32 storage keeps the fixture small
    # and is far below the 1e-6 tolerance these vectors are checked at
    out = {k: (v.astype(np.float32) if v.dtype == np.float64 else v)
           for k, v in out.items()}
    np.savez_compressed(os.path.join(HERE, "golden_filter.npz"), **out)


def make_bp():
    n, nrow = 96, 72
    sino, ang, _ = phantom.ellipse_sinogram(21, nrow, n, 47.5, photons=1e4)
    f = rec.apply_ramp_filter(sino, None, "hann", None, "edge")
    f = np.float32(f)
    out = {"filtered": f, "angles": ang}
    for cen in (47.5, 45.3, 52.0):
        for ep in (False, True):
            out[_key("bp", cen, int(ep))] = rec.back_projection_cpu(
                f, np.float32(ang), np.float32(cen), ep)
    # odd width, 360-degree angles including the endpoint
    n2, nrow2 = 81, 61
    ang2 = np.deg2rad(np.linspace(0.0, 360.0, nrow2))
    s2, _, _ = phantom.ellipse_sinogram(22, nrow2, n2, 40.0, photons=1e4,
                                        angles=ang2)
    f2 = np.float32(rec.apply_ramp_filter(s2, None, "hann", None, "edge"))
    out["filtered_odd"] = f2
    out["angles_odd"] = ang2
    for ep in (False, True):
        out[_key("bpodd", 40.0, int(ep))] = rec.back_projection_cpu(
            f2, np.float32(ang2), np.float32(40.0), ep)
    np.savez_compressed(os.path.join(HERE, "golden_bp.npz"), **out)


def make_recon():
    n, nrow = 96, 73
    sino, ang, _ = phantom.ellipse_sinogram(31, nrow, n, 47.5, photons=1e4)
    trans = np.exp(-sino).astype(np.float32)  # transmission, for apply_log
    trans[5, 10] = 0.0
    trans[9, 3] = -0.5
    out = {"sino": sino, "trans": trans, "angles": ang}
    for name, fn in (("fbp", rec.fbp_reconstruction),
                     ("bpf", rec.bpf_reconstruction)):
        for ratio in (1.0, 0.0, None):
            out[_key(name, "2d", ratio)] = fn(sino.copy(), 47.5, angles=ang,
                                              ratio=ratio, apply_log=False,
                                              gpu=False)
        out[_key(name, "2d", "defang")] = fn(sino.copy(), 45.3,
                                             apply_log=False, gpu=False)
        out[_key(name, "2d", "nofilter", "reflect")] = fn(
            sino.copy(), 47.5, angles=ang, filter_name=None, pad=10,
            pad_mode="reflect", apply_log=False, gpu=False)
        t = trans.copy()
        with warnings.catch_warnings(record=True) as caught:
            warnings.simplefilter("always")
            out[_key(name, "2d", "log")] = fn(t, 47.5, angles=ang,
                                              apply_log=True, gpu=False)
        out[_key(name, "2d", "log", "warned")] = np.array(len(caught) > 0)
        out[_key(name, "2d", "log", "mutated")] = t
        s3 = np.stack([sino, 0.5 * sino, sino[:, ::-1].copy()], axis=1)
        out[_key(name, "3d", 0.0)] = fn(s3.copy(), 47.5, angles=ang,
                                        ratio=0.0, apply_log=False,
                                        gpu=False, ncore=1)
        out[_key(name, "3d1", 1.0)] = fn(s3[:, :1].copy(), 47.5, angles=ang,
                                         apply_log=False, gpu=False, ncore=1)
    out["s3"] = np.stack([sino, 0.5 * sino, sino[:, ::-1].copy()], axis=1)
    dtypes = {k: str(v.dtype) for k, v in out.items()}
    out = {k: (v.astype(np.float32) if v.dtype == np.float64 and
               k.startswith(("fbp", "bpf")) else v) for k, v in out.items()}
    out["dtypes"] = np.array(repr(dtypes))
    np.savez_compressed(os.path.join(HERE, "golden_recon.npz"), **out)


def make_reference_test_fixture():
    """The reference's own unit-test phantom (test_reconstruction.py:50-65)."""
    size = 64
    mat = np.zeros((size + 1, size + 1), dtype=np.float32)
    mat[20:40, 30:45] = np.float32(1.0)
    mat = ndi.gaussian_filter(mat, 2.0)
    sino_360 = np.zeros((73, size + 1), dtype=np.float32)
    angles = np.linspace(0.0, 360.0, len(sino_360), dtype=np.float32)
    for i, angle in enumerate(angles):
        sino_360[i] = np.sum(ndi.rotate(mat, -angle, reshape=False), axis=0)
    out = {"mat": mat, "sino_360": sino_360, "angles_deg": angles}
    out["fbp_180"] = rec.fbp_reconstruction(sino_360[:37].copy(), 32,
                                            apply_log=False, gpu=False)
    out["bpf_180"] = rec.bpf_reconstruction(sino_360[:37].copy(), 32,
                                            apply_log=False, gpu=False)
    np.savez_compressed(os.path.join(HERE, "golden_unittest.npz"), **out)


def make_center():
    """Centre search by slice metrics (reconstruction.py:1212-1458).

    The reference's own pre-steps on fixed inputs (Gaussian smoothing along
    the detector, linear zoom, the two metrics), the metric of every
    candidate centre of ``_find_center_based_slice_metric`` and the centre
    chosen by ``find_center_based_slice_metric`` (FBP and BPF methods).
    """
    entropy = getattr(rec, "__calculate_histogram_entropy")
    sharp = getattr(rec, "__calculate_edge_sharpness")
    n, nrow, cen = 96, 91, 46.3
    sino, ang, _ = phantom.ellipse_sinogram(41, nrow, n, cen, photons=2e4)
    trans = np.exp(-sino).astype(np.float32)
    trans[7, 11] = 0.0
    out = {"sino": sino, "trans": trans, "angles": ang,
           "center": np.float64(cen)}
    # pre-steps
    for sigma in (1, 2, 3.5):
        out[_key("gauss", sigma)] = ndi.gaussian_filter1d(sino, sigma, axis=1)
    narrow = sino[:, 40:45].copy()
    out["narrow"] = narrow
    out[_key("gauss", "narrow", 2)] = ndi.gaussian_filter1d(narrow, 2,
                                                             axis=1)
    for z in (0.5, 0.8, 0.33):
        out[_key("zoom", z)] = ndi.zoom(sino, z, order=1, mode="nearest")
        out[_key("zoom", "angles", z)] = ndi.zoom(np.tile(ang, (1, 1)),
                                                  (1.0, z))[0]
    # metrics of fixed images (the reconstruction at the true centre)
    img = rec.fbp_reconstruction(sino.copy(), cen, angles=ang,
                                 apply_log=False, gpu=False)
    nmin, nmax = np.min(img), np.max(img)
    img1 = np.clip((img - nmin) / (nmax - nmin), 0, 1)
    out["metric_img"] = img
    out[_key("metric", "entropy")] = np.float64(
        entropy(img1, ssig.windows.boxcar(7)))
    out[_key("metric", "sharpness")] = np.float64(sharp(img))
    # every candidate's metric
    f = rec._find_center_based_slice_metric
    cases = {
        "fbp_entropy": dict(metric="entropy", method="fbp", sigma=2,
                            ratio=1.0),
        "fbp_sharp": dict(metric="sharpness", method="fbp", sigma=0,
                          ratio=1.0),
        "fbp_entropy_r0": dict(metric="entropy", method="fbp", sigma=1,
                               ratio=0.0),
        "fbp_entropy_nomask": dict(metric="entropy", method="fbp", sigma=2,
                                   ratio=None),
        "bpf_entropy": dict(metric="entropy", method="bpf", sigma=2,
                            ratio=1.0),
        "bpf_sharp": dict(metric="sharpness", method="bpf", sigma=2,
                          ratio=1.0),
    }
    for name, kw in cases.items():
        cs, ms = f(sino.copy(), cen - 3, cen + 3, 0.5, angles=ang,
                   apply_log=False, gpu=False, ncore=1, return_metric=True,
                   **kw)
        out[_key("list", name, "centers")] = cs
        out[_key("list", name, "metrics")] = ms
    cs, ms = f(trans.copy(), cen - 2, cen + 2, 1.0, angles=ang,
               apply_log=True, gpu=False, ncore=1, return_metric=True)
    out[_key("list", "log", "centers")] = cs
    out[_key("list", "log", "metrics")] = ms
    # integer counts: scipy smooths them into the same integer type,
    # truncated toward zero, before the -log
    counts = np.uint16(trans * 40000.0)
    out["counts"] = counts
    out[_key("gauss", "u16", 2)] = ndi.gaussian_filter1d(counts, 2, axis=1)
    cs, ms = f(counts.copy(), cen - 2, cen + 2, 1.0, angles=ang, sigma=2,
               apply_log=True, gpu=False, ncore=1, return_metric=True)
    out[_key("list", "u16", "centers")] = cs
    out[_key("list", "u16", "metrics")] = ms
    # chosen centres of the two-pass search
    g = rec.find_center_based_slice_metric
    finds = {
        "z1": dict(zoom=1.0, angles=ang),
        "z05": dict(zoom=0.5, angles=ang),
        "z08_default_angles": dict(zoom=0.8, angles=None),
        "sharp": dict(zoom=1.0, angles=ang, metric="sharpness"),
        "bpf": dict(zoom=1.0, angles=ang, method="bpf"),
        "r0": dict(zoom=1.0, angles=ang, radius=0.0),
    }
    for name, kw in finds.items():
        out[_key("find", name)] = np.float64(g(
            sino.copy(), cen - 6, cen + 6, step=0.25, gpu=False,
            apply_log=False, ncore=1, **kw))
    np.savez_compressed(os.path.join(HERE, "golden_center.npz"), **out)


def make_vertical():
    """Vertical slices (algotom/rec/vertrec.py): the back-projectors, the
    slice geometry and the three chunked reconstructions, CPU path."""
    import algotom.rec.vertrec as vrec
    nproj, height, width, cen = 73, 10, 64, 31.7
    ang = np.deg2rad(np.linspace(0.0, 180.0, nproj))
    att = np.zeros((nproj, height, width), np.float32)
    for i in range(height):
        att[:, i, :] = phantom.ellipse_sinogram(60 + i, nproj, width, cen,
                                                photons=None, angles=ang)[0]
    trans = np.exp(-att).astype(np.float32)
    rng = np.random.default_rng(7)
    flat = (1.0 + 0.05 * rng.random((height, width))).astype(np.float32)
    dark = (0.01 * rng.random((height, width))).astype(np.float32)
    raw = (trans * (flat - dark) + dark).astype(np.float32)
    out = {"att": att, "trans": trans, "angles": ang, "flat": flat,
           "dark": dark, "raw": raw, "center": np.float64(cen)}
    for w in (64, 65, 9):
        for idx, alpha in ((0, 0.0), (w // 2, 30.0), (w - 1, 45.0),
                           (w // 3, 60.0), (w // 2, 90.0), (1, 135.0),
                           (w - 2, 150.0), (w // 2, 180.0)):
            xs, ys = vrec._get_points_single_line(idx, alpha, w)
            out[_key("pts", w, idx, alpha, "x")] = xs
            out[_key("pts", w, idx, alpha, "y")] = ys
    lines = ((32, 0.0), (20, 30.0), (40, 60.0), (10, 90.0), (50, 150.0))
    for idx, alpha in lines:
        xs, ys = vrec._get_points_single_line(idx, alpha, width)
        for ep in (False, True):
            out[_key("vbp", idx, alpha, ep)] = vrec.vertical_back_projection_cpu(
                att, ang, xs, ys, cen, edge_pad=ep)
    xm, ym = vrec._get_points_multiple_lines(20, 44, 45.0, width, 8)
    out["xm"], out["ym"] = xm, ym
    for ep in (False, True):
        out[_key("vbpchunk", ep)] = vrec.vertical_back_projection_cpu_chunk(
            att, ang, xm, ym, cen, edge_pad=ep)
    common = dict(gpu=False, show_progress=False, ncore=1)
    rec_cases = {
        "after": dict(),
        "before": dict(ramp_filter="before"),
        "none": dict(ramp_filter=None),
        "crop_range": dict(crop=(1, 2, 3, 4), proj_start=2, proj_stop=70,
                           chunk_size=16, masking=True),
        "flat": dict(flat_field=flat, dark_field=dark, chunk_size=20,
                     ramp_filter="before", pad=10, pad_mode="reflect"),
        "alpha": dict(alpha=70.0, filter_name="hamming", chunk_size=None),
    }
    for name, kw in rec_cases.items():
        src = raw if "flat_field" in kw else trans
        a = ang[2:70] if "proj_stop" in kw else ang
        out[_key("vrec", name)] = vrec.vertical_reconstruction(
            src.copy(), 30, cen - (3 if "crop" in kw else 0), angles=a,
            **kw, **common)
    out["vrec_multi"] = vrec.vertical_reconstruction_multiple(
        trans.copy(), 20, 40, cen, alpha=45.0, step_index=5, angles=ang,
        chunk_size=25, **common)
    out["vrec_diff"] = vrec.vertical_reconstruction_different_angles(
        trans.copy(), [10, 30, 50], [0.0, 60.0, 120.0], cen, angles=ang,
        ramp_filter="before", chunk_size=30, masking=True, **common)
    bad = trans.copy()
    bad[5, 3, 7] = 0.0
    bad[40, 8, 20] = -1.0
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        out["vrec_log"] = vrec.vertical_reconstruction(
            bad, 30, cen, angles=ang, chunk_size=30, **common)
    out["vrec_log_warnings"] = np.array([str(w.message) for w in caught
                                         if "logarithm" in str(w.message)])
    out["vrec_log_mutated"] = bad
    np.savez_compressed(os.path.join(HERE, "golden_vertical.npz"), **out)


def make_vcenter():
    """Centre search on a vertical slice (find_center_vertical_slice,
    algotom/rec/vertrec.py:1264-1383), CPU path, and the projection
    smoothing it starts with."""
    import scipy.ndimage as ndi
    import algotom.rec.vertrec as vrec
    nproj, height, width, cen = 73, 10, 64, 31.7
    ang = np.deg2rad(np.linspace(0.0, 180.0, nproj))
    att = np.zeros((nproj, height, width), np.float32)
    for i in range(height):
        att[:, i, :] = phantom.ellipse_sinogram(60 + i, nproj, width, cen,
                                                photons=None, angles=ang)[0]
    trans = np.exp(-att).astype(np.float32)
    rng = np.random.default_rng(11)
    tall = rng.random((3, 70, 40)).astype(np.float32)
    out = {"trans": trans, "angles": ang, "tall": tall}
    for sg in (3, 1.5, 0.7):
        out[_key("smooth", sg)] = ndi.gaussian_filter(trans, (0, sg, sg))
        out[_key("smooth_tall", sg)] = ndi.gaussian_filter(tall, (0, sg, sg))
    common = dict(gpu=False, show_progress=False, ncore=1, return_metric=True)
    cases = {
        "entropy": dict(),
        "sharpness": dict(metric="sharpness"),
        "autocorr": dict(metric="autocorrelation"),
        "entropy_before": dict(ramp_filter="before", sigma=1.5),
        "sharp_nomask": dict(metric="sharpness", masking=False, sigma=0,
                             alpha=30.0, slice_index=20),
        "entropy_invert": dict(invert_metric=True, chunk_size=16, sigma=0.7),
        "autocorr_angles": dict(metric="autocorrelation", alpha=60.0,
                                slice_index=40, angles=ang, chunk_size=None),
    }
    for name, kw in cases.items():
        kw = dict(kw)
        idx = kw.pop("slice_index", 32)
        cs, ms = vrec.find_center_vertical_slice(
            trans.copy(), idx, 28.0, 35.0, step=0.5, **kw, **common)
        out[_key("vc", name, "centers")] = cs
        out[_key("vc", name, "metrics")] = ms
    cs, ms = vrec.find_center_vertical_slice(trans.copy(), 32, 28, 35,
                                             step=1, metric="sharpness",
                                             **common)
    out["vc_int_centers"], out["vc_int_metrics"] = cs, ms
    out["vc_best"] = vrec.find_center_vertical_slice(
        trans.copy(), 32, 28.0, 35.0, step=0.5, gpu=False,
        show_progress=False, ncore=1)
    bad = trans.copy()
    bad[5, 3, 7] = 0.0
    bad[40, 8, 20] = -1.0
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        cs, ms = vrec.find_center_vertical_slice(
            bad, 32, 29.0, 34.0, step=1.0, sigma=0, metric="sharpness",
            **common)
    out["vc_log_metrics"] = ms
    # integer counts: each smoothing pass is truncated toward zero.  (Not
    # with apply_log=False and the "after" filter: the reference's CPU
    # back-projector then interpolates the uint16 counts in uint16, and a
    # negative difference wraps around -- slices of ~1e18.)
    counts = np.uint16(trans * 40000.0)
    out["counts"] = counts
    for sg in (3, 1.5):
        out[_key("smooth_u16", sg)] = ndi.gaussian_filter(counts,
                                                          (0, sg, sg))
    for name, kw in (("u16_entropy", dict()),
                     ("u16_sharp_before_nolog",
                      dict(metric="sharpness", apply_log=False, sigma=1.5,
                           ramp_filter="before"))):
        cs, ms = vrec.find_center_vertical_slice(
            counts.copy(), 32, 28.0, 35.0, step=0.5, **kw, **common)
        out[_key("vc", name, "centers")] = cs
        out[_key("vc", name, "metrics")] = ms
    out["vc_log_warnings"] = np.array([str(w.message) for w in caught
                                       if "logarithm" in str(w.message)])
    out["vc_log_mutated"] = bad
    # the reference's own search test data (tests/test_rec/test_vertrec.py:
    # 52-81, 498-539): a 3-D phantom of three cut squares, projected by
    # rotation over 180 degrees; centre 30
    import algotom.util.utility as util
    w, h = 61, 40
    mat = util.make_circle_mask(w, 0.8)
    for rad, i_s, j_s in ((10, 30, 20), (5, 20, 30), (5, 20, 50)):
        mat[i_s:i_s + rad, j_s:j_s + rad] = 0
    mat = ndi.gaussian_filter(mat, 1)
    vol = np.zeros((h, w, w), dtype=np.float32)
    vol[1:] = mat
    ang360 = np.linspace(0.0, 360.0, 91, dtype=np.float32)
    projs = np.zeros((91, h, w), dtype=np.float32)
    for i, a in enumerate(ang360):
        projs[i] = np.sum(ndi.rotate(vol, -a, axes=(1, 2), order=1,
                                     reshape=False), axis=1)
    projs = projs[:46] + 1
    out["cube_projs"] = projs
    for metric in ("autocorrelation", "entropy", "sharpness"):
        cs, ms = vrec.find_center_vertical_slice(
            projs.copy(), w // 2, 25, 39, step=1.0, metric=metric,
            invert_metric=True, masking=False, **common)
        out[_key("cube", metric, "centers")] = cs
        out[_key("cube", metric, "metrics")] = ms

    def get_negative(mat, n=2):
        return np.abs(np.mean(mat[mat < 0.0])) ** n
    cs, ms = vrec.find_center_vertical_slice(
        projs.copy(), w // 2, 25, 39, step=1.0, invert_metric=True,
        metric_function=get_negative, n=2, **common)
    out["cube__custom__centers"], out["cube__custom__metrics"] = cs, ms
    np.savez_compressed(os.path.join(HERE, "golden_vcenter.npz"), **out)


def make_conversion():
    """360-degree conversions (algotom/prep/conversion.py:43-454) and the
    scipy sub-pixel shift they call."""
    import algotom.prep.conversion as conv
    from scipy.ndimage import shift as ndi_shift
    nrow, ncol = 181, 64
    ang = np.linspace(0.0, 2.0 * np.pi, nrow)
    out = {}
    for cor in (50.3, 12.7, 45.5, 20.0):
        att = phantom.ellipse_sinogram(70, nrow, ncol, cor, photons=None,
                                       angles=ang)[0]
        trans = np.exp(-0.2 * att).astype(np.float32)
        out[_key("att", cor)] = att
        out[_key("trans", cor)] = trans
        sino, c = conv.extend_sinogram(trans.copy(), cor)
        out[_key("extend", cor)], out[_key("extend", cor, "cor")] = sino, c
        sino, c = conv.extend_sinogram(att.copy(), cor, apply_log=False)
        out[_key("extend_nolog", cor)] = sino
        sino, c = conv.convert_sinogram_360_to_180(att.copy(), cor)
        out[_key("to180", cor)], out[_key("to180", cor, "cor")] = sino, c
        sino, _ = conv.convert_sinogram_360_to_180(att.copy(), cor,
                                                   norm=False,
                                                   total_width=2 * ncol)
        out[_key("to180_nonorm_wide", cor)] = sino
    att = out[_key("att", 50.3)]
    sino, c = conv.extend_sinogram(att.copy(), (27.4, 1), apply_log=False)
    out["extend_tuple"], out["extend_tuple_cor"] = sino, c
    sino, c = conv.convert_sinogram_360_to_180(att.copy(), (27.4, 1))
    out["to180_tuple"], out["to180_tuple_cor"] = sino, c
    s180 = out[_key("att", 20.0)][:91]
    for center in (30.4, 33.0, 18.25):
        out[_key("to360", center)] = conv.convert_sinogram_180_to_360(
            s180.copy(), center)
    out["s180"] = s180
    rng = np.random.default_rng(5)
    x = rng.standard_normal((12, 97)).astype(np.float32)
    out["shift_x"] = x
    for sh in (0.3, -0.45, 11.3, -15.6, 40.2):
        out[_key("shift", sh)] = ndi_shift(x, (0, sh), mode="nearest")
    np.savez_compressed(os.path.join(HERE, "golden_conversion.npz"), **out)


def make_visual():
    """The visual centre searches (reconstruction.py:1461-1533,
    vertrec.py:1431-1535), CPU path: the file names each writes and the
    images read back from them."""
    import shutil
    import tempfile
    from PIL import Image
    import algotom.rec.vertrec as vrec

    def read_folder(base):
        names = sorted(os.listdir(base))
        imgs = [np.array(Image.open(os.path.join(base, n))) for n in names]
        return np.array(names), np.stack(imgs)

    n, nrow, cen = 96, 91, 46.3
    sino, ang, _ = phantom.ellipse_sinogram(41, nrow, n, cen, photons=2e4)
    trans = np.exp(-sino).astype(np.float32)
    out = {"trans": trans, "angles": ang}
    cases = {
        "fbp_zoom": dict(start=42.0, stop=50.0, step=1.5, zoom=0.5),
        "fbp_angles": dict(start=44.0, stop=48.0, step=1.0, zoom=1.0,
                           angles=ang, ratio=0.0),
        "bpf": dict(start=45.0, stop=47.0, step=0.5, zoom=1.0,
                    method="bpf"),
        "dfi_zoom": dict(start=44.0, stop=47.0, step=1.0, zoom=0.5,
                         method="dfi", filter_name=None),
    }
    tmp = tempfile.mkdtemp()
    try:
        for name, kw in cases.items():
            base = rec.find_center_visual_slices(trans.copy(), tmp, **kw,
                                                 gpu=False, ncore=1)
            out[_key("vis", name, "folder")] = np.array(
                os.path.basename(base.rstrip("/")))
            out[_key("vis", name, "names")], out[_key("vis", name, "imgs")] = \
                read_folder(base)
        w, h = 61, 40
        mat = util.make_circle_mask(w, 0.8)
        for rad, i_s, j_s in ((10, 30, 20), (5, 20, 30), (5, 20, 50)):
            mat[i_s:i_s + rad, j_s:j_s + rad] = 0
        mat = ndi.gaussian_filter(mat, 1)
        vol = np.zeros((h, w, w), dtype=np.float32)
        vol[1:] = mat
        ang360 = np.linspace(0.0, 360.0, 91, dtype=np.float32)
        projs = np.zeros((91, h, w), dtype=np.float32)
        for i, a in enumerate(ang360):
            projs[i] = np.sum(ndi.rotate(vol, -a, axes=(1, 2), order=1,
                                         reshape=False), axis=1)
        projs = projs[:46] + 1
        out["cube_projs"] = projs
        vcases = {
            "after": dict(start=28.0, stop=31.0, step=1.0),
            "before_nomask": dict(start=29.0, stop=30.5, step=0.5,
                                  ramp_filter="before", masking=False,
                                  alpha=30.0),
        }
        for name, kw in vcases.items():
            base = vrec.find_center_visual_vertical_slices(
                projs.copy(), tmp, w // 2, **kw, gpu=False, ncore=1,
                display=False)
            out[_key("vvis", name, "names")], out[_key("vvis", name, "imgs")] \
                = read_folder(base)
    finally:
        shutil.rmtree(tmp)
    np.savez_compressed(os.path.join(HERE, "golden_visual.npz"), **out)


def make_dfi():
    """DFI reconstruction (reconstruction.py:687-907)."""
    nrow, ncol, cen = 181, 96, 47.3
    ang = np.linspace(0.0, np.pi, nrow)
    sino = phantom.ellipse_sinogram(80, nrow, ncol, cen, photons=2e4,
                                    angles=ang)[0]
    out = {"sino": sino, "angles": ang, "center": np.float64(cen)}
    r, t = rec.generate_mapping_coordinate(97 + 48, nrow, 97 + 48, 97 + 48)
    out["map_r"], out["map_theta"] = r, t
    f = rec.dfi_reconstruction
    out["dfi_default"] = f(sino.copy(), cen, apply_log=False)
    out["dfi_angles"] = f(sino.copy(), cen, angles=ang, apply_log=False)
    off = ang + 0.1
    out["dfi_angles_offset"] = f(sino.copy(), cen, angles=off,
                                 apply_log=False)
    out["dfi_angles_desc"] = f(sino[::-1].copy(), cen, angles=ang[::-1],
                               apply_log=False)
    ang360 = np.linspace(0.0, 2 * np.pi, 2 * nrow - 1)
    s360 = np.concatenate([sino, sino[-2::-1, ::-1]], axis=0)
    out["sino360"] = s360
    out["dfi_360"] = f(s360.copy(), cen, angles=ang360, apply_log=False)
    out["dfi_r0_nofilter"] = f(sino.copy(), cen, ratio=0.0, filter_name=None,
                               apply_log=False)
    out["dfi_reflect_pad05"] = f(sino.copy(), cen, ratio=None,
                                 pad_mode="reflect", pad_rate=0.5,
                                 apply_log=False)
    odd = sino[:, :95].copy()
    out["sino_odd"] = odd
    out["dfi_odd"] = f(odd.copy(), 46.8, apply_log=False)
    trans = np.exp(-sino).astype(np.float32)
    trans[10, 20] = 0.0
    out["trans"] = trans
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        out["dfi_log"] = f(trans.copy(), cen)
    out["dfi_log_warned"] = np.array(
        any("logarithm" in str(w.message) for w in caught))
    s3 = np.stack([sino, 0.5 * sino], axis=1)
    out["dfi_3d"] = f(s3.copy(), cen, apply_log=False, ncore=1)
    np.savez_compressed(os.path.join(HERE, "golden_dfi.npz"), **out)


GENERATORS = {"windows": make_windows, "filter": make_filter, "bp": make_bp,
              "recon": make_recon, "unittest": make_reference_test_fixture,
              "center": make_center, "vertical": make_vertical,
              "vcenter": make_vcenter, "visual": make_visual,
              "conversion": make_conversion, "dfi": make_dfi}

if __name__ == "__main__":
    # python make_golden.py [name ...]  (default: every fixture)
    for name in (sys.argv[1:] or list(GENERATORS)):
        GENERATORS[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
