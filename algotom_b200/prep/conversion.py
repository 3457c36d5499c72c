"""Drop-in replacement of algotom's 360-degree sinogram conversions.

Same names, signatures, results and errors as ``algotom/prep/conversion.py``
(algotom 1.6.0) for ``make_weight_matrix`` (``:43-73``), ``stitch_image``
(``:76-144``), ``convert_sinogram_360_to_180`` (``:318-364``),
``convert_sinogram_180_to_360`` (``:367-392``) and ``extend_sinogram``
(``:395-454``).  The row work -- ``-log``, the sub-pixel cubic-spline shift
(scipy's ``ndimage.shift`` with ``mode="nearest"``), the overlap ramp, edge
padding and scaling -- runs in the sm_100a kernels ``atb_shift_rows`` and
``atb_extend_rows``; the stitching of two shifted halves is device array
arithmetic in the reference's float32 order.  NumPy in, NumPy out; torch
CUDA tensors stay on the device, so a half-acquisition sinogram can go
straight into :func:`algotom_b200.rec.reconstruction.fbp_reconstruction`
with the returned centre.
"""
import numpy as np
import torch

from .. import _native as nat
from ..rec import reconstruction as R


def _overlap_side(cor, ncol):
    if isinstance(cor, tuple):
        return cor
    if cor <= (ncol - 1.0) * 0.5:
        return 2 * cor + 1, 0
    return 2 * (ncol - cor) - 1, 1


def _shift_rows(t, shift, flip=False):
    """float32 ``scipy.ndimage.shift(t, (0, shift), mode="nearest")`` of a
    2-D CUDA tensor (mirrored left-right first when ``flip``)."""
    nrow, ncol = t.shape
    out = torch.empty((nrow, ncol), dtype=torch.float32, device=t.device)
    nat.call("atb_shift_rows", t.data_ptr(), t.stride(0), nrow, ncol,
             float(shift), int(bool(flip)), out.data_ptr(), out.stride(0),
             R._stream_ptr(t.device))
    return out


def _finish(t, is_np):
    return t.cpu().numpy() if is_np else t


def make_weight_matrix(mat1, mat2, overlap, side):
    """Linear-ramp weights for stitching; ``conversion.py:43-73``.  Host
    arrays shaped like ``mat1`` / ``mat2`` (tensors in, tensors out)."""
    tens = isinstance(mat1, torch.Tensor)
    shape1, shape2 = tuple(mat1.shape), tuple(mat2.shape)
    overlap = int(np.floor(overlap))
    wei_mat1 = np.ones(shape1, dtype=np.float32)
    wei_mat2 = np.ones(shape2, dtype=np.float32)
    list_down = np.linspace(1.0, 0.0, overlap)
    list_up = 1.0 - list_down
    if side == 1:
        wei_mat1[:, -overlap:] = np.float32(list_down)
        wei_mat2[:, :overlap] = np.float32(list_up)
    else:
        wei_mat2[:, -overlap:] = np.float32(list_down)
        wei_mat1[:, :overlap] = np.float32(list_up)
    if tens:
        return (torch.from_numpy(wei_mat1).to(mat1.device),
                torch.from_numpy(wei_mat2).to(mat2.device))
    return wei_mat1, wei_mat2


def stitch_image(mat1, mat2, overlap, side, wei_mat1=None, wei_mat2=None,
                 norm=True, total_width=None):
    """Stitch two images with a linear ramp over ``overlap`` columns on
    ``side`` of image 1; ``conversion.py:76-144``."""
    t1, is_np = R._to_device(mat1)
    t2, _ = R._to_device(mat2, t1.device)
    (nrow1, ncol1), (nrow2, ncol2) = t1.shape, t2.shape
    overlap_int = int(np.round(overlap + 1.0e-3))
    sub_pixel = overlap - overlap_int
    if sub_pixel != 0.0:
        if side == 1:
            t1, t2 = _shift_rows(t1, sub_pixel), _shift_rows(t2, -sub_pixel)
        else:
            t1, t2 = _shift_rows(t1, -sub_pixel), _shift_rows(t2, sub_pixel)
    if nrow1 != nrow2:
        raise ValueError("Two images are not at the same height!!!")
    if (wei_mat1 is None) or (wei_mat2 is None):
        wei_mat1, wei_mat2 = make_weight_matrix(t1.cpu(), t2.cpu(),
                                                overlap_int, side)
    w1 = torch.as_tensor(np.asarray(wei_mat1), device=t1.device)
    w2 = torch.as_tensor(np.asarray(wei_mat2), device=t1.device)
    total_width0 = ncol1 + ncol2 - overlap_int
    if (total_width is None) or (total_width < total_width0):
        total_width = total_width0
    comb = torch.zeros((nrow1, total_width0), dtype=torch.float32,
                       device=t1.device)
    if side == 1:
        if norm is True:
            f1 = t1[:, -overlap_int:].mean(dtype=torch.float64).float()
            f2 = t2[:, :overlap_int].mean(dtype=torch.float64).float()
            t2 = t2 * f1 / f2
        comb[:, 0:ncol1] = (t1 * w1).float()
        comb[:, (ncol1 - overlap_int):total_width0] += (t2 * w2).float()
    else:
        if norm is True:
            f2 = t2[:, -overlap_int:].mean(dtype=torch.float64).float()
            f1 = t1[:, :overlap_int].mean(dtype=torch.float64).float()
            t2 = t2 * f1 / f2
        comb[:, 0:ncol2] = (t2 * w2).float()
        comb[:, (ncol2 - overlap_int):total_width0] += (t1 * w1).float()
    if total_width > total_width0:
        comb = torch.cat([comb, comb[:, -1:].expand(
            nrow1, total_width - total_width0)], dim=1)
    return _finish(comb, is_np)


def convert_sinogram_360_to_180(sino_360, cor, wei_mat1=None, wei_mat2=None,
                                norm=True, total_width=None):
    """Convert a 360-degree sinogram (offset rotation axis) to a 180-degree
    one; ``conversion.py:318-364``.  Returns (sinogram, centre)."""
    t, is_np = R._to_device(sino_360)
    nrow, ncol = t.shape
    nrow_180 = nrow // 2 + 1
    top = t[0:nrow_180, :]
    bot = torch.flip(t[-nrow_180:, :], dims=[1])
    overlap, side = _overlap_side(cor, ncol)
    out = stitch_image(top, bot, overlap, side, wei_mat1=wei_mat1,
                       wei_mat2=wei_mat2, norm=norm, total_width=total_width)
    overlap_int = int(np.round(overlap + 1.0e-3))
    cor = ncol - overlap_int / 2.0 - 0.5
    return _finish(out, is_np), cor


def convert_sinogram_180_to_360(sino_180, center):
    """Convert a 180-degree sinogram to a 360-degree one;
    ``conversion.py:367-392``."""
    t, is_np = R._to_device(sino_180)
    nrow, ncol = t.shape
    shift_x = (ncol - 1.0) / 2.0 - center
    flip = _shift_rows(_shift_rows(t, shift_x), -shift_x, flip=True)
    return _finish(torch.cat([t, flip[1:]], dim=0), is_np)


def extend_sinogram(sino_360, cor, apply_log=True):
    """Extend a 360-degree sinogram with an offset rotation axis for direct
    reconstruction; ``conversion.py:395-454``.  Returns (sinogram, centre):
    ``2 ncol - overlap`` columns, the overlap ramped, the far side padded
    with the edge samples, doubled."""
    t, is_np = R._to_device(sino_360)
    nrow, ncol = t.shape
    overlap, side = _overlap_side(cor, ncol)
    overlap_int = int(np.round(overlap + 1.0e-3))
    sub_pixel = overlap - overlap_int
    shift = 0.0 if sub_pixel == 0.0 else (sub_pixel if side == 1
                                          else -sub_pixel)
    out = torch.empty((nrow, 2 * ncol - overlap_int), dtype=torch.float32,
                      device=t.device)
    nat.call("atb_extend_rows", t.data_ptr(), t.stride(0), nrow, ncol,
             int(bool(apply_log)), float(shift), overlap_int, int(side),
             out.data_ptr(), out.stride(0), R._stream_ptr(t.device))
    cor = ncol - overlap_int / 2.0 - 0.5
    return _finish(out, is_np), cor
