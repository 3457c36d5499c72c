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
