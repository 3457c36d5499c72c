"""Drop-in replacement of algotom's DFI reconstruction.

``dfi_reconstruction`` and ``generate_mapping_coordinate`` of
``algotom/rec/reconstruction.py`` (algotom 1.6.0, ``:687-907``): same
signatures, errors, warnings and output dtypes.  The direct Fourier
inversion runs on the device:

1. the sinogram is padded by one edge column when its width is even and
   centred with the cubic-spline sub-pixel shift of
   ``scipy.ndimage.shift(mode="nearest")`` (``atb_shift_rows``); given
   ``angles``, a 360-degree scan is folded to 180 degrees and the rows are
   rotated to start at angle 0 with the same spline along the angle axis
   (``mode="wrap"``, ``atb_spline_prefilter`` then the spline taps);
2. the detector axis is padded (NumPy's modes, device index maps) and, with
   ``apply_log``, values <= 0 are set to 1 (with the reference's warning)
   before ``-log``;
3. every row is transformed (library FFT, FP64) and windowed;
4. the polar spectrum is turned into quintic B-spline coefficients along
   both axes (``atb_spline_prefilter``, the prefilter's impulse response as
   a parallel FIR) and regridded onto the Cartesian
   frequency grid with the unit-circle mask (``atb_dfi_regrid``);
5. an inverse 2-D transform (library FFT, FP64), crop and circle mask.

FP64 from step 3 on; the reference runs its row transform in the input's
float32 precision, so results agree to ~1e-7.  ``ncore`` is accepted and
ignored.
"""
import warnings

import numpy as np
import torch

from .. import _native as nat
from . import reconstruction as R
from . import windows as win
from .padding import pad_rows


def generate_mapping_coordinate(width_sino, height_sino, width_rec,
                                height_rec):
    """Sinogram-space (radius, angle) coordinates of the Cartesian frequency
    grid; ``reconstruction.py:687-728``.  float32 (r_mat, theta_mat).  (The
    device regridding forms the same coordinates per pixel.)"""
    xcenter = (width_rec - 1.0) * 0.5
    ycenter = (height_rec - 1.0) * 0.5
    r_max = np.floor(min(xcenter, ycenter))
    xlist = (np.flipud(np.arange(width_rec)) - xcenter)
    ylist = (np.arange(height_rec) - ycenter)
    x_mat, y_mat = np.meshgrid(xlist, ylist)
    r_mat = np.float32(np.clip(np.sqrt(x_mat ** 2 + y_mat ** 2), 0, r_max))
    theta_mat = np.pi + np.arctan2(y_mat, x_mat)
    r_mat[theta_mat > np.pi] *= -1
    r_mat = np.float32(np.clip(r_mat + r_max, 0, width_sino - 1))
    theta_mat[theta_mat > np.pi] -= np.pi
    theta_mat = np.float32(theta_mat * (height_sino - 1.0) / np.pi)
    return r_mat, theta_mat


def _prefilter(t, axis, order, boundary):
    """B-spline coefficients of a contiguous float64 / complex128 2-D CUDA
    tensor along ``axis``, in a new tensor (boundary 0: half-sample
    symmetric, 1: whole-sample symmetric)."""
    h, w = t.shape
    ncomp = 2 if t.is_complex() else 1
    if axis == 1:
        lines, line_stride, es, n = h, w * ncomp, ncomp, w
    else:
        lines, line_stride, es, n = w, ncomp, w * ncomp, h
    out = torch.empty_like(t)
    nat.call("atb_spline_prefilter", t.data_ptr(), out.data_ptr(),
             line_stride, es, lines, ncomp, n, order, boundary,
             R._stream_ptr(t.device))
    return out


def _bspline3(u):
    a = u.abs()
    return torch.where(a < 1, 2.0 / 3.0 - a * a + a * a * a / 2.0,
                       torch.where(a < 2, (2.0 - a) ** 3 / 6.0,
                                   torch.zeros_like(a)))


def _shift_cols_wrap(t32, s):
    """float32 ``scipy.ndimage.shift(t32, (s, 0), mode="wrap")``: cubic
    spline along the rows' axis with whole-sample symmetric coefficients,
    coordinates wrapped with period n - 1 and mirrored taps."""
    n = t32.shape[0]
    c = _prefilter(t32.to(torch.float64).contiguous(), 0, 3, 1)
    cc = torch.arange(n, dtype=torch.float64, device=t32.device) - s
    sz = n - 1
    if sz > 0:
        cc = torch.where(cc < 0, cc + sz * (torch.floor(-cc / sz) + 1), cc)
        cc = torch.where(cc > n - 1, cc - sz * torch.floor(cc / sz), cc)
    f = torch.floor(cc).to(torch.int64)
    out = torch.zeros(c.shape, dtype=torch.float64, device=c.device)
    for m in range(-1, 3):
        idx = f + m
        if n > 1:
            p = 2 * (n - 1)
            r = torch.remainder(idx, p)
            idx = torch.where(r >= n, p - r, r)
        else:
            idx = torch.zeros_like(idx)
        out += _bspline3(cc - (f + m).to(torch.float64))[:, None] * c[idx]
    return out.to(torch.float32)


def _handle_angles(t, angles):
    """``__dfi_handle_angles`` (reconstruction.py:731-749) on the device."""
    nrow = t.shape[0]
    if len(angles) != nrow:
        raise ValueError("!!! Number of angles is not the same as the row "
                         "number of the sinogram !!!")
    angles = np.asarray(angles, dtype=np.float64)
    t_ang = np.sum(np.abs(np.diff(angles * 180.0 / np.pi)))
    if abs(t_ang - 360) < 10:
        nrow = nrow // 2 + 1
        t = (t[:nrow] + torch.flip(t[-nrow:], dims=[1])) / 2
    step = np.mean(np.abs(np.diff(angles)))
    b_ang = angles[0] - (angles[0] // (2 * np.pi)) * (2 * np.pi)
    sino_360 = torch.cat([t[:nrow - 1], torch.flip(t, dims=[1])], dim=0)
    t = _shift_cols_wrap(sino_360, b_ang / step)[:nrow]
    if angles[-1] < angles[0]:
        t = torch.flip(t, dims=[0, 1])
    return t


def _circle_mask(width, ratio, device):
    c = width // 2
    radius = ratio * c
    ax = torch.arange(-c, width - c, device=device, dtype=torch.float64)
    return (ax[None, :] ** 2 + ax[:, None] ** 2 <= radius * radius).to(
        torch.float64)


def _dfi_slice(s, window, pad, ncol):
    """Steps 3-5 for one prepared float32 [nrow, ncol2] CUDA sinogram;
    returns the float64 [ncol, ncol] image (cropped at ``pad``).  The
    regridding writes its grid in ifftshift order and the final fftshift
    and crop are one index gather, so the 2-D shifts cost no extra pass."""
    nrow, w = s.shape
    x = s.to(torch.float64)
    f = torch.fft.fftshift(torch.fft.fft(torch.fft.ifftshift(x, dim=1),
                                         dim=1), dim=1)
    if window is not None:
        f = f * window
    f = _prefilter(_prefilter(f.contiguous(), 0, 5, 0), 1, 5, 0)
    reg = torch.empty((w, w), dtype=torch.complex128, device=s.device)
    nat.call("atb_dfi_regrid", f.data_ptr(), nrow, w, reg.data_ptr(),
             R._stream_ptr(s.device))
    y = torch.fft.ifft2(reg).real
    # fftshift(y)[k] = y[(k - w // 2) mod w], rows and columns pad..pad+ncol
    idx = torch.remainder(torch.arange(pad, pad + ncol, device=s.device)
                          - w // 2, w)
    return y.index_select(0, idx).index_select(1, idx)


def dfi_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       filter_name="hann", pad_rate=0.25, pad_mode="edge",
                       apply_log=True, ncore=None):
    """DFI (direct Fourier inversion) of a 2-D sinogram or a 3-D stack
    (slices on axis 1); ``reconstruction.py:818-907``.  Returns float64
    (float32 with ``filter_name=None``, as the reference), [ncol, ncol] or
    [ncol, nslice, ncol]."""
    input_3d = len(sinogram.shape) == 3
    nrow, ncol = sinogram.shape[0], sinogram.shape[-1]
    if center < 0 or center >= ncol:
        raise ValueError("Center is out of the range [0, {}]".format(ncol - 1))
    if ncol / nrow > 5.0:
        warnings.warn("!!!Sinogram is significantly undersampled!!! "
                      "Considering to use the 'upsample_sinogram' method "
                      "before reconstruction!")
    if pad_mode not in nat.PAD_MODES:
        raise ValueError("pad_mode %r is not supported" % (pad_mode,))
    t, is_np = R._to_device(sinogram)
    slices = [t] if t.dim() == 2 else [t[:, k, :] for k in range(t.shape[1])]
    prepared = []
    pad = 0
    for s in slices:
        if ncol % 2 == 0:
            s = torch.cat([s, s[:, -1:]], dim=1)
        ncol1 = s.shape[1]
        xshift = (ncol1 - 1) / 2.0 - center
        pad = int(pad_rate * ncol1)
        s = _shift_rows(s.contiguous(), xshift)
        if angles is not None:
            s = _handle_angles(s, angles)
        prepared.append(pad_rows(s, pad, pad_mode))
    stack = torch.stack(prepared)
    if apply_log is True:
        bad = stack <= 0.0
        if bool(bad.any()):
            warnings.warn("!!!Applying logarithm is enabled but "
                          "there are values <= 0.0 in the data!!!")
            stack = stack.masked_fill(bad, 1.0)
        stack = -torch.log(stack)
    nrow2, ncol2 = stack.shape[1], stack.shape[2]
    window = None
    if filter_name is not None:
        window = torch.from_numpy(win.make_smoothing_window(
            filter_name, ncol2)).to(t.device)
    mask = None
    if ratio is not None:
        if ratio == 0.0:
            ratio = min(center, ncol - center) / (0.5 * ncol)
        mask = _circle_mask(ncol, ratio, t.device)
    out = []
    for s in stack:
        r = _dfi_slice(s, window, pad, ncol)
        out.append(r * mask if mask is not None else r)
    rec = torch.stack(out, dim=1) if len(out) > 1 or input_3d else out[0]
    dtype = torch.float64 if filter_name is not None else torch.float32
    rec = rec.to(dtype)
    return rec.cpu().numpy() if is_np else rec


def _shift_rows(t, shift):
    from ..prep.conversion import _shift_rows as shift_rows
    return shift_rows(t, shift)
