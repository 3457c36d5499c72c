"""Direct Fourier inversion (reconstruction.py:687-907).

CPU tests pin the FP64 oracle (``oracle/dfi_oracle.py``) to the reference's
outputs (``tests/golden/golden_dfi.npz``; the reference's row transform is
float32, so agreement is ~1e-7) and the host coordinate map bit-exactly.
GPU tests hold the device path, through the C ABI, to the reference's
outputs (1e-6 relative L2), its dtypes, errors and warnings, the spline
prefilter to the oracle (1e-12), and port the reference's own centre-search
test, which uses DFI (test_reconstruction.py:242-272).
"""
import warnings

import numpy as np
import pytest

from algotom_b200 import _native as nat
from oracle import dfi_oracle as D
from oracle import fbp_oracle as O

TOL = 1e-6


def _cases(g):
    sino, ang, cen = g["sino"], g["angles"], float(g["center"])
    return {
        "dfi_default": dict(sinogram=sino, center=cen),
        "dfi_angles": dict(sinogram=sino, center=cen, angles=ang),
        "dfi_angles_offset": dict(sinogram=sino, center=cen, angles=ang + 0.1),
        "dfi_angles_desc": dict(sinogram=sino[::-1].copy(), center=cen,
                                angles=ang[::-1].copy()),
        "dfi_360": dict(sinogram=g["sino360"], center=cen,
                        angles=np.linspace(0.0, 2 * np.pi, 361)),
        "dfi_r0_nofilter": dict(sinogram=sino, center=cen, ratio=0.0,
                                filter_name=None),
        "dfi_reflect_pad05": dict(sinogram=sino, center=cen, ratio=None,
                                  pad_mode="reflect", pad_rate=0.5),
        "dfi_odd": dict(sinogram=g["sino_odd"], center=46.8),
    }


NAMES = ["dfi_default", "dfi_angles", "dfi_angles_offset", "dfi_angles_desc",
         "dfi_360", "dfi_r0_nofilter", "dfi_reflect_pad05", "dfi_odd"]


# ------------------------------------------------------------- CPU
def test_mapping_coordinates_bit_exact(golden):
    from algotom_b200.rec import reconstruction as R
    g = golden("dfi")
    for fn in (R.generate_mapping_coordinate, D.mapping_coordinates):
        r, t = fn(145, 181, 145, 145)
        assert np.array_equal(r, g["map_r"]) and np.array_equal(
            t, g["map_theta"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(golden, name):
    g = golden("dfi")
    got = D.dfi_reconstruction(apply_log=False, **_cases(g)[name])
    assert O.rel_l2(got, g[name]) < TOL


def test_abi_argument_errors():
    lib = nat.load()
    one = 1
    two = 2
    assert lib.atb_spline_prefilter(None, two, 8, 1, 2, 1, 8, 5, 0,
                                    None) == -1
    assert lib.atb_spline_prefilter(one, one, 8, 1, 2, 1, 8, 5, 0,
                                    None) == -1  # in place
    assert lib.atb_spline_prefilter(one, two, 8, 1, 2, 3, 8, 5, 0,
                                    None) == -1
    assert lib.atb_spline_prefilter(one, two, 8, 1, 2, 1, 8, 4, 0,
                                    None) == -1
    assert lib.atb_spline_prefilter(one, two, 8, 1, 2, 1, 8, 5, 2,
                                    None) == -1
    assert lib.atb_spline_prefilter(one, two, 8, 3, 2, 1, 8, 5, 0,
                                    None) == -1  # neither axis contiguous
    assert lib.atb_dfi_regrid(None, 8, 8, one, None) == -1
    assert lib.atb_dfi_regrid(one, 8, 50000, one, None) == -3
    assert b"too large" in lib.atb_last_error()
    # own transforms: M = the power of two >= 2 w - 1, at most 8192
    assert lib.atb_dfi_fft_length(3841) == 8192
    assert lib.atb_dfi_fft_length(5) == 16
    assert lib.atb_dfi_fft_length(4097) == -3
    assert lib.atb_dfi_fft_length(1) == -1
    assert lib.atb_dfi_rows(one, 8, 0, 4, 1, 8, 2, 10, 0, None, None, one,
                            one, one, one, two, 12, 0, None) == -1
    assert b"pad_mode" in lib.atb_last_error()
    assert lib.atb_dfi_rows(None, 8, 0, 4, 1, 8, 2, 0, 0, None, None, one,
                            one, one, one, two, 12, 0, None) == -1
    assert lib.atb_dfi_inverse_workspace(15, 8, 2) == 2 * 15 * 8 * 16
    assert lib.atb_dfi_inverse_workspace(15, 16, 1) == -1
    assert lib.atb_dfi_inverse(one, 15, 0, 9, 1, 15, 4, 12, -1.0, one, one,
                               one, one, two, 12, 0, 0, two, 1 << 20,
                               None) == -1  # crop beyond the width
    assert lib.atb_dfi_inverse(one, 15, 0, 9, 1, 15, 3, 8, -1.0, one, one,
                               one, one, two, 8, 0, 0, two, 100,
                               None) == -1  # workspace too small
    assert b"workspace" in lib.atb_last_error()
    assert lib.atb_wrap_shift_rows(one, 8, 0, 5, 1, 8, 0.5, 6, 0, two, 8, 0,
                                   None) == -1  # nout > m
    assert lib.atb_wrap_shift_rows(one, 8, 0, 5, 1, 8, float("nan"), 5, 0,
                                   two, 8, 0, None) == -1
    assert lib.atb_shift_rows_ext(one, 8, 4, 9, 8, 0.5, two, 8,
                                  None) == -1  # fewer columns out than in


def test_center_error():
    from algotom_b200.rec import reconstruction as R
    with pytest.raises(ValueError, match="Center is out of the range"):
        R.dfi_reconstruction(np.ones((9, 16), np.float32), 16.0)


# ------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("order", [3, 5])
@pytest.mark.parametrize("boundary", ["reflect", "mirror"])
def test_spline_prefilter_matches_oracle(cuda, order, boundary):
    import torch
    from algotom_b200.rec import dfi
    rng = np.random.default_rng(order)
    x = rng.standard_normal((13, 40)) + 1j * rng.standard_normal((13, 40))
    bnd = 0 if boundary == "reflect" else 1
    for axis in (0, 1):
        t = torch.as_tensor(x, device="cuda").contiguous()
        got = dfi._prefilter(t, axis, order, bnd).cpu().numpy()
        src = x if axis == 1 else x.T
        ref = D.spline_filter1d(src, order, boundary)
        ref = ref if axis == 1 else ref.T
        assert np.max(np.abs(got - ref)) < 1e-12 * np.max(np.abs(ref))
    xr = rng.standard_normal((7, 3))
    t = torch.as_tensor(xr, device="cuda").contiguous()
    got = dfi._prefilter(t, 0, order, bnd).cpu().numpy()
    ref = D.spline_filter1d(xr.T, order, boundary).T
    assert np.max(np.abs(got - ref)) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_wrap_shift_matches_oracle(cuda):
    import torch
    from algotom_b200.rec import dfi
    rng = np.random.default_rng(9)
    x = rng.standard_normal((19, 11)).astype(np.float32)
    for s in (0.0, 0.3, 2.6, -1.4, 7.2):
        got = dfi._shift_cols_wrap(torch.as_tensor(x, device="cuda"),
                                   s).cpu().numpy()
        ref = D.shift_cols_wrap(x, s)
        assert np.max(np.abs(got.astype(np.float64) - ref)) <= \
            np.max(np.spacing(np.abs(ref)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_dfi_matches_reference(cuda, golden, name):
    from algotom_b200.rec import reconstruction as R
    g = golden("dfi")
    kw = _cases(g)[name]
    got = R.dfi_reconstruction(kw.pop("sinogram").copy(), apply_log=False,
                               **kw)
    ref = g[name]
    assert got.dtype == ref.dtype and got.shape == ref.shape
    assert O.rel_l2(got, ref) < TOL


@pytest.mark.gpu
def test_dfi_log_3d_and_warnings(cuda, golden):
    import torch
    from algotom_b200.rec import reconstruction as R
    g = golden("dfi")
    cen = float(g["center"])
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        got = R.dfi_reconstruction(g["trans"].copy(), cen)
    warned = any("logarithm" in str(w.message) for w in caught)
    assert warned == bool(g["dfi_log_warned"])
    assert O.rel_l2(got, g["dfi_log"]) < TOL
    s3 = np.stack([g["sino"], 0.5 * g["sino"]], axis=1)
    got = R.dfi_reconstruction(s3, cen, apply_log=False)
    assert got.shape == g["dfi_3d"].shape
    assert O.rel_l2(got, g["dfi_3d"]) < TOL
    t = R.dfi_reconstruction(torch.as_tensor(g["sino"], device="cuda"), cen,
                             apply_log=False)
    assert isinstance(t, torch.Tensor) and t.is_cuda
    assert O.rel_l2(t.cpu().numpy(), g["dfi_default"]) < TOL
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        R.dfi_reconstruction(np.ones((10, 64), np.float32), 31.5,
                             apply_log=False)
    assert any("undersampled" in str(w.message) for w in caught)


@pytest.mark.gpu
def test_reference_centre_search_tests_with_dfi(cuda, golden):
    """Port of test_reconstruction.py:242-272 (method "dfi")."""
    from algotom_b200.rec import reconstruction as R
    g = golden("unittest")
    sino_180 = g["sino_360"][:37]
    angles2 = g["angles_deg"][:37]
    center = 32
    f = R.find_center_based_slice_metric
    got = f(sino_180.copy(), center - 2, center + 2, step=0.25, radius=2,
            zoom=0.8, method="dfi", gpu=False, angles=np.deg2rad(angles2),
            ratio=1.0, filter_name="hann", apply_log=False, ncore=1,
            sigma=1, metric_function=None)
    assert abs(got - center) < 0.1
    got = f(sino_180.copy(), center - 2, center + 2, step=0.25,
            metric="sharpness", radius=2, zoom=1.0, method="dfi", gpu=False,
            angles=None, ratio=1.0, filter_name="hann", apply_log=False,
            ncore=1, sigma=0, metric_function=None)
    assert abs(got - center) <= 0.25

    def get_negative(mat, n=2):
        return np.abs(np.mean(mat[mat < 0.0])) ** n

    got = f(sino_180.copy(), center - 2, center + 2, step=0.25, radius=2,
            zoom=1.0, method="dfi", gpu=False, angles=None, ratio=1.0,
            filter_name="hann", apply_log=False, ncore=None, sigma=1,
            metric_function=get_negative, n=2)
    assert abs(got - center) < 0.1


@pytest.mark.gpu
def test_dfi_row_transform_matches_numpy(cuda):
    """atb_dfi_rows at the benchmark's width (2561 + 2 x 640 = 3841 =
    23 x 167, M = 8192): padding, pairs of rows per transform (an odd row
    count leaves one alone), strided slices, window; FP64 to 1e-12 (no
    -log here: its float32 rounding would be all the test saw)."""
    import torch
    from algotom_b200.rec import dfi
    from algotom_b200.rec import reconstruction as R
    rng = np.random.default_rng(5)
    nrow, nslice, n, pad = 5, 2, 2561, 640
    w = n + 2 * pad
    x = rng.random((nrow, nslice, n)).astype(np.float32) + 0.1
    win = rng.random(w)
    t = torch.as_tensor(x, device="cuda")
    wt = torch.as_tensor(win, device="cuda")
    chirp, tw, bfwd, binv = dfi._fft_tables(w, t.device)
    out = torch.empty((nrow, nslice, w), dtype=torch.complex128,
                      device="cuda")
    nat.call("atb_dfi_rows", t.data_ptr(), nslice * n, n, nrow, nslice, n,
             pad, nat.PAD_MODES["edge"], 0, wt.data_ptr(), None,
             chirp.data_ptr(), tw.data_ptr(), bfwd.data_ptr(),
             binv.data_ptr(), out.data_ptr(), nslice * w, w,
             R._stream_ptr())
    got = out.cpu().numpy()
    for k in range(nslice):
        s = np.pad(x[:, k, :], ((0, 0), (pad, pad)), mode="edge")
        ref = np.fft.fftshift(np.fft.fft(np.fft.ifftshift(
            s.astype(np.float64), axes=1)), axes=1) * win
        err = np.abs(got[:, k, :] - ref).max() / np.abs(ref).max()
        assert err < 1e-12, err


@pytest.mark.gpu
@pytest.mark.parametrize("mode", sorted(nat.PAD_MODES))
def test_dfi_pad_modes_with_log(cuda, mode):
    """Every numpy pad mode through the fused padding of atb_dfi_rows, with
    -log and values <= 0 (the reference's warning), against the FP64
    oracle (np.pad itself)."""
    from algotom_b200.rec import reconstruction as R
    rng = np.random.default_rng(len(mode))
    nrow, ncol = 31, 24
    sino = np.exp(-rng.random((nrow, ncol)) * 2.0).astype(np.float32)
    sino[3, 5] = 0.0
    sino[7, 0] = -1.0
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        got = R.dfi_reconstruction(sino.copy(), 11.6, pad_mode=mode,
                                   pad_rate=0.5)
    assert any("logarithm" in str(w.message) for w in caught)
    ref = D.dfi_reconstruction(sino, 11.6, pad_mode=mode, pad_rate=0.5,
                               apply_log=True)
    assert O.rel_l2(got, ref) < TOL


@pytest.mark.gpu
def test_dfi_own_transforms_match_library_fft(cuda):
    """The benchmark slice (1801 x 2560, padded to 3841) through this
    library's transforms and through the library-FFT path of wider rows:
    same spline and regridding kernels, independent transforms."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.rec import dfi
    from algotom_b200.rec import reconstruction as R
    nrow, ncol, cen = 1801, 2560, 1278.3
    ang = np.linspace(0.0, np.pi, nrow, endpoint=False)
    s, _, _ = phantom.ellipse_sinogram(2000, nrow, ncol, cen, angles=ang)
    got = R.dfi_reconstruction(torch.as_tensor(s, device="cuda"), cen,
                               apply_log=False)
    ncol1 = ncol + 1
    pad = int(0.25 * ncol1)
    sh = torch.empty((nrow, 1, ncol1), dtype=torch.float32, device="cuda")
    t = torch.as_tensor(s, device="cuda")
    nat.call("atb_shift_rows_ext", t.data_ptr(), ncol, nrow, ncol, ncol1,
             (ncol1 - 1) / 2.0 - cen, sh.data_ptr(), ncol1, R._stream_ptr())
    w = ncol1 + 2 * pad
    ref = torch.empty((ncol, ncol), dtype=torch.float64, device="cuda")
    radius = ncol // 2
    dfi._dfi_wide(sh, ref, pad, ncol, "edge", False,
                  dfi._window("hann", w, t.device), float(radius * radius))
    err = (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item()
    assert err < 1e-10, err
