"""360-degree sinogram conversions (algotom/prep/conversion.py).

CPU tests pin the FP64 oracle (``oracle/conversion_oracle.py``) to vectors
produced by the reference (``tests/golden/golden_conversion.npz``): the
cubic-spline sub-pixel shift bit-exactly, the conversions to 1e-7 relative
L2 (the reference runs them in float32).  GPU tests hold the device path,
through the C ABI, to the reference's outputs: the shift to one float32
rounding step, the conversions to 1e-6 relative L2, the returned centres
exactly.  (The device prefilter is the FIR of the recursive filter's
impulse response; the two differ by ~1e-18 of the row's largest value, so
the float32 step is counted from 1e-10 of that value upwards: outputs that
are near-cancellations, e.g. a zero padded region next to data, may differ
from scipy's by ~1e-18 absolute.)
"""
import numpy as np
import pytest

from algotom_b200 import _native as nat
from oracle import conversion_oracle as C
from oracle import fbp_oracle as O

CORS = (50.3, 12.7, 45.5, 20.0)
SHIFTS = (0.3, -0.45, 11.3, -15.6, 40.2)
CENTERS_180 = (30.4, 33.0, 18.25)
TOL = 1e-6


# ------------------------------------------------------------- CPU
@pytest.mark.parametrize("sh", SHIFTS)
def test_oracle_spline_shift_bit_exact(golden, sh):
    g = golden("conversion")
    assert np.array_equal(C.shift_rows(g["shift_x"], sh), g["shift__%s" % sh])


@pytest.mark.parametrize("cor", CORS)
def test_oracle_conversions(golden, cor):
    g = golden("conversion")
    e, c = C.extend_sinogram(g["trans__%s" % cor], cor)
    assert O.rel_l2(e, g["extend__%s" % cor]) < 1e-7
    assert c == float(g["extend__%s__cor" % cor])
    e, _ = C.extend_sinogram(g["att__%s" % cor], cor, apply_log=False)
    assert O.rel_l2(e, g["extend_nolog__%s" % cor]) < 1e-7
    t, c = C.convert_sinogram_360_to_180(g["att__%s" % cor], cor)
    assert O.rel_l2(t, g["to180__%s" % cor]) < 1e-7
    assert c == float(g["to180__%s__cor" % cor])
    t, _ = C.convert_sinogram_360_to_180(g["att__%s" % cor], cor, norm=False,
                                         total_width=128)
    assert O.rel_l2(t, g["to180_nonorm_wide__%s" % cor]) < 1e-7


@pytest.mark.parametrize("center", CENTERS_180)
def test_oracle_180_to_360(golden, center):
    g = golden("conversion")
    got = C.convert_sinogram_180_to_360(g["s180"], center)
    assert O.rel_l2(got, g["to360__%s" % center]) < 1e-12


def test_weight_matrix_matches_oracle():
    from algotom_b200.prep import conversion as PC
    a, b = np.ones((3, 20), np.float32), np.ones((3, 17), np.float32)
    for side in (0, 1):
        for ov in (1, 2, 7, 17):
            got = PC.make_weight_matrix(a, b, ov, side)
            ref = C.make_weight_matrix(a, b, ov, side)
            assert all(np.array_equal(x, y) and x.dtype == np.float32
                       for x, y in zip(got, ref))


def test_abi_argument_errors():
    lib = nat.load()
    one = 1
    assert lib.atb_shift_rows(None, 8, 2, 8, 0.5, 0, one, 8, None) == -1
    assert lib.atb_shift_rows(one, 8, 2, 20000, 0.5, 0, one, 8, None) == -3
    assert lib.atb_shift_rows(one, 8, 2, 8, float("inf"), 0, one, 8,
                              None) == -1
    assert lib.atb_extend_rows(one, 8, 2, 8, 1, 0.0, 0, 1, one, 8,
                               None) == -1  # no overlap
    assert lib.atb_extend_rows(one, 8, 2, 8, 1, 0.0, 9, 1, one, 8,
                               None) == -1  # overlap wider than the row
    assert lib.atb_extend_rows(one, 8, 2, 8, 1, 0.0, 3, 2, one, 8,
                               None) == -1  # unknown side
    assert b"side" in lib.atb_last_error()


# ------------------------------------------------------------- GPU
def _f32_steps(a, b):
    """Largest difference in units of float32 rounding of the reference,
    values below 1e-10 of its largest magnitude counted at that level."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    mag = np.maximum(np.abs(b), 1e-10 * np.abs(b).max())
    ulp = np.spacing(mag.astype(np.float32)).astype(np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(ulp, 1e-45)))


@pytest.mark.gpu
@pytest.mark.parametrize("sh", SHIFTS)
def test_shift_rows_matches_scipy(cuda, golden, sh):
    import torch
    from algotom_b200.prep import conversion as PC
    g = golden("conversion")
    x = torch.as_tensor(g["shift_x"], device="cuda")
    got = PC._shift_rows(x, sh).cpu().numpy()
    assert _f32_steps(got, g["shift__%s" % sh]) <= 1.0
    # mirrored input
    got = PC._shift_rows(x, sh, flip=True).cpu().numpy()
    ref = C.shift_rows(np.ascontiguousarray(g["shift_x"][:, ::-1]), sh)
    assert _f32_steps(got, ref) <= 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("cor", CORS)
def test_extend_and_360_to_180_match_reference(cuda, golden, cor):
    from algotom_b200.prep import conversion as PC
    g = golden("conversion")
    trans, att = g["trans__%s" % cor], g["att__%s" % cor]
    keep = trans.copy()
    e, c = PC.extend_sinogram(trans, cor)
    ref = g["extend__%s" % cor]
    assert e.dtype == np.float32 and e.shape == ref.shape
    assert O.rel_l2(e, ref) < TOL and c == float(g["extend__%s__cor" % cor])
    assert np.array_equal(trans, keep)  # the input is not modified
    e, _ = PC.extend_sinogram(att, cor, apply_log=False)
    assert O.rel_l2(e, g["extend_nolog__%s" % cor]) < TOL
    t, c = PC.convert_sinogram_360_to_180(att, cor)
    ref = g["to180__%s" % cor]
    assert t.dtype == np.float32 and t.shape == ref.shape
    assert O.rel_l2(t, ref) < TOL and c == float(g["to180__%s__cor" % cor])
    t, _ = PC.convert_sinogram_360_to_180(att, cor, norm=False,
                                          total_width=128)
    assert O.rel_l2(t, g["to180_nonorm_wide__%s" % cor]) < TOL


@pytest.mark.gpu
def test_tuple_centre_and_180_to_360(cuda, golden):
    from algotom_b200.prep import conversion as PC
    g = golden("conversion")
    att = g["att__50.3"]
    e, c = PC.extend_sinogram(att, (27.4, 1), apply_log=False)
    assert O.rel_l2(e, g["extend_tuple"]) < TOL
    assert c == float(g["extend_tuple_cor"])
    t, c = PC.convert_sinogram_360_to_180(att, (27.4, 1))
    assert O.rel_l2(t, g["to180_tuple"]) < TOL
    assert c == float(g["to180_tuple_cor"])
    for center in CENTERS_180:
        got = PC.convert_sinogram_180_to_360(g["s180"], center)
        ref = g["to360__%s" % center]
        assert got.shape == ref.shape
        assert _f32_steps(got, ref) <= 1.0


@pytest.mark.gpu
def test_extend_feeds_fbp_on_device(cuda, golden):
    """A half-acquisition sinogram extended on the device reconstructs like
    the oracle's extension through the FP64 FBP restatement."""
    import torch
    from algotom_b200.prep import conversion as PC
    from algotom_b200.rec import reconstruction as R
    g = golden("conversion")
    trans = g["trans__50.3"]
    ang = np.linspace(0.0, 2.0 * np.pi, trans.shape[0])
    e, c = PC.extend_sinogram(torch.as_tensor(trans, device="cuda"), 50.3)
    assert isinstance(e, torch.Tensor) and e.is_cuda
    rec = R.fbp_reconstruction(e, c, angles=ang, apply_log=False)
    ref_sino, _ = C.extend_sinogram(trans, 50.3)
    ref = O.fbp_reconstruction(ref_sino.astype(np.float32), c, angles=ang,
                               apply_log=False)
    assert O.rel_l2(rec.cpu().numpy(), ref) < 1e-5
