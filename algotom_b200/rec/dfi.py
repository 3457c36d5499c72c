"""Drop-in replacement of algotom's DFI reconstruction.

``dfi_reconstruction`` and ``generate_mapping_coordinate`` of
``algotom/rec/reconstruction.py`` (algotom 1.6.0, ``:687-907``): same
signatures, errors, warnings and output dtypes.  The direct Fourier
inversion runs on the device, every slice of a stack in the same launches:

1. every row is padded by one edge column when the width is even and
   centred with the cubic-spline sub-pixel shift of
   ``scipy.ndimage.shift(mode="nearest")`` (``atb_shift_rows_ext``);
2. given ``angles``, a 360-degree scan is folded to 180 degrees and the
   rows are rotated to start at angle 0 with the same spline along the
   angle axis (``mode="wrap"``: ``atb_dfi_angle_stack``,
   ``atb_spline_prefilter``, ``atb_wrap_shift_rows``);
3. padding with NumPy's modes, ``-log`` (values <= 0 counted for the
   reference's warning), the centred row transform and the window, two
   rows per FP64 Bluestein transform (``atb_dfi_rows``);
4. quintic B-spline coefficients of the polar spectrum along both axes
   (``atb_spline_prefilter``);
5. regridding onto the Cartesian frequency grid row by row, inverse 2-D
   transform, crop, ``1 / w^2`` and circle mask (``atb_dfi_inverse``).

The transforms are this library's own (``csrc/dfi_fft.cu``) for padded
widths up to 4096 (2730 detector columns at the default ``pad_rate``);
wider rows take the library FFT for steps 3 and 5 (``_dfi_wide``).  FP64
from step 3 on; the reference runs its row transform in the input's
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

_SPECTRA_BYTES = 4 << 30   # polar spectra (+ their coefficients) per launch
_TABLES = {}
_WINDOWS = {}


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


def _shift_cols_wrap(t32, s):
    """float32 ``scipy.ndimage.shift(t32, (s, 0), mode="wrap")`` of a 2-D
    CUDA tensor: cubic-spline coefficients along the rows (whole-sample
    symmetric), then the wrapped taps of ``atb_wrap_shift_rows``."""
    m, n = t32.shape
    c = _prefilter(t32.to(torch.float64).contiguous(), 0, 3, 1)
    out = torch.empty((m, n), dtype=torch.float32, device=t32.device)
    nat.call("atb_wrap_shift_rows", c.data_ptr(), n, 0, m, 1, n, float(s),
             m, 0, out.data_ptr(), n, 0, R._stream_ptr(t32.device))
    return out


def _fft_tables(w, device):
    """(chirp, twiddle, bfwd, binv) device tables of the width-w Bluestein
    transforms, made once per (device, w).  The chirp's phase pi m^2 / w is
    reduced exactly (m^2 mod 2w in integers) before the trigonometry."""
    key = (device.index, w)
    tab = _TABLES.get(key)
    if tab is None:
        M = nat.call("atb_dfi_fft_length", w)
        m = np.arange(w, dtype=np.int64)
        chirp = np.exp(1j * (np.pi * ((m * m) % (2 * w)) / w))
        k = np.arange(M, dtype=np.float64)
        tw = np.exp(-2j * np.pi * k / M)
        chirp = torch.from_numpy(chirp).to(device)
        tw = torch.from_numpy(tw).to(device)
        bfwd = torch.empty(M, dtype=torch.complex128, device=device)
        binv = torch.empty(M, dtype=torch.complex128, device=device)
        nat.call("atb_dfi_fft_setup", w, chirp.data_ptr(), tw.data_ptr(),
                 bfwd.data_ptr(), binv.data_ptr(), R._stream_ptr(device))
        tab = _TABLES[key] = (chirp, tw, bfwd, binv)
    return tab


def _window(filter_name, w, device):
    key = (device.index, filter_name, w)
    t = _WINDOWS.get(key)
    if t is None:
        t = _WINDOWS[key] = torch.from_numpy(
            win.make_smoothing_window(filter_name, w)).to(device)
    return t


def _own_transform(w):
    return 2 <= w and 2 * w - 1 <= 8192


def _angle_rows(sh, angles):
    """``__dfi_handle_angles`` (``reconstruction.py:731-749``) of every
    slice of the [nrow, nslice, ncol1] float32 stack at once."""
    nrow, nslice, ncol1 = sh.shape
    if len(angles) != nrow:
        raise ValueError("!!! Number of angles is not the same as the row "
                         "number of the sinogram !!!")
    angles = np.asarray(angles, dtype=np.float64)
    t_ang = np.sum(np.abs(np.diff(angles * 180.0 / np.pi)))
    fold = abs(t_ang - 360) < 10
    n1 = nrow // 2 + 1 if fold else nrow
    step = np.mean(np.abs(np.diff(angles)))
    b_ang = angles[0] - (angles[0] // (2 * np.pi)) * (2 * np.pi)
    m = 2 * n1 - 1
    dev, st = sh.device, R._stream_ptr(sh.device)
    lines = nslice * ncol1
    stack = torch.empty((m, nslice, ncol1), dtype=torch.float64, device=dev)
    nat.call("atb_dfi_angle_stack", sh.data_ptr(), lines, ncol1, nrow,
             nslice, ncol1, int(fold), stack.data_ptr(), lines, ncol1, st)
    coef = torch.empty_like(stack)
    nat.call("atb_spline_prefilter", stack.data_ptr(), coef.data_ptr(), 1,
             lines, lines, 1, m, 3, 1, st)
    del stack
    out = torch.empty((n1, nslice, ncol1), dtype=torch.float32, device=dev)
    nat.call("atb_wrap_shift_rows", coef.data_ptr(), lines, ncol1, m,
             nslice, ncol1, float(b_ang / step), n1,
             int(angles[-1] < angles[0]), out.data_ptr(), lines, ncol1, st)
    return out


def _dfi_own(sh, out, pad, ncol, pad_mode, apply_log, window, mask_r2):
    """Steps 3-5 on this library's transforms: the prepared float32
    [nrow, nslice, ncol1] stack into ``out`` ([ncol, nslice, ncol] or
    [ncol, ncol]), slices in groups whose spectra fit the budget.
    Returns the number of padded values <= 0 (with ``apply_log``)."""
    nrow, nslice, ncol1 = sh.shape
    w = ncol1 + 2 * pad
    dev, st = sh.device, R._stream_ptr(sh.device)
    chirp, tw, bfwd, binv = _fft_tables(w, dev)
    # (the row-wise prefilter takes up to 65535 lines per launch)
    group = max(1, min(nslice, _SPECTRA_BYTES // (2 * 16 * nrow * w),
                       65535 // nrow))
    f32 = int(out.dtype == torch.float32)
    ors = out.stride(0)
    oss = out.stride(1) if out.dim() == 3 else 0
    counter = torch.empty(1, dtype=torch.int32, device=dev)
    bad = 0
    spec = torch.empty((nrow, group, w), dtype=torch.complex128, device=dev)
    tmp = torch.empty_like(spec)
    wbytes = nat.call("atb_dfi_inverse_workspace", w, ncol, group)
    ws = torch.empty(wbytes, dtype=torch.uint8, device=dev)
    for k0 in range(0, nslice, group):
        g = min(group, nslice - k0)
        src = sh[:, k0:k0 + g]
        nat.call("atb_dfi_rows", src.data_ptr(), nslice * ncol1, ncol1,
                 nrow, g, ncol1, pad, nat.PAD_MODES[pad_mode],
                 int(apply_log),
                 window.data_ptr() if window is not None else None,
                 counter.data_ptr() if apply_log else None,
                 chirp.data_ptr(), tw.data_ptr(), bfwd.data_ptr(),
                 binv.data_ptr(), spec.data_ptr(), g * w, w, st)
        if apply_log:
            bad += int(counter.item())
        # quintic coefficients along the angles, then along the frequencies
        nat.call("atb_spline_prefilter", spec.data_ptr(), tmp.data_ptr(), 2,
                 2 * g * w, g * w, 2, nrow, 5, 0, st)
        nat.call("atb_spline_prefilter", tmp.data_ptr(), spec.data_ptr(),
                 2 * w, 2, nrow * g, 2, w, 5, 0, st)
        nat.call("atb_dfi_inverse", spec.data_ptr(), g * w, w, nrow, g, w,
                 pad, ncol, float(mask_r2), chirp.data_ptr(), tw.data_ptr(),
                 bfwd.data_ptr(), binv.data_ptr(),
                 out.data_ptr() + k0 * oss * out.element_size(), ors, oss,
                 f32, ws.data_ptr(), wbytes, st)
    return bad


def _dfi_wide(sh, out, pad, ncol, pad_mode, apply_log, window, mask_r2):
    """Steps 3-5 for padded widths beyond the own transforms' 4096: padding
    and ``-log`` as tensor operations, the row transform and the inverse 2-D
    transform through the library FFT, the spline and regridding kernels as
    above."""
    nrow, nslice, ncol1 = sh.shape
    w = ncol1 + 2 * pad
    bad = 0
    c = ncol // 2
    ax = torch.arange(-c, ncol - c, device=sh.device, dtype=torch.float64)
    mask = None if mask_r2 < 0 else \
        (ax[None, :] ** 2 + ax[:, None] ** 2 <= mask_r2).to(torch.float64)
    idx = torch.remainder(torch.arange(pad, pad + ncol, device=sh.device)
                          - w // 2, w)
    for k in range(nslice):
        s = pad_rows(sh[:, k, :], pad, pad_mode)
        if apply_log:
            neg = s <= 0.0
            bad += int(neg.sum())
            s = -torch.log(s.masked_fill(neg, 1.0))
        x = s.to(torch.float64)
        f = torch.fft.fftshift(torch.fft.fft(torch.fft.ifftshift(x, dim=1),
                                             dim=1), dim=1)
        if window is not None:
            f = f * window
        f = _prefilter(_prefilter(f.contiguous(), 0, 5, 0), 1, 5, 0)
        reg = torch.empty((w, w), dtype=torch.complex128, device=sh.device)
        nat.call("atb_dfi_regrid", f.data_ptr(), nrow, w, reg.data_ptr(),
                 R._stream_ptr(sh.device))
        y = torch.fft.ifft2(reg).real.index_select(0, idx).index_select(1,
                                                                        idx)
        if mask is not None:
            y = y * mask
        if out.dim() == 3:
            out[:, k, :] = y
        else:
            out.copy_(y)
    return bad


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
    if input_3d:
        t = t.contiguous()
    nslice = t.shape[1] if input_3d else 1
    dev, st = t.device, R._stream_ptr(t.device)
    ncol1 = ncol + 1 if ncol % 2 == 0 else ncol
    xshift = (ncol1 - 1) / 2.0 - center
    pad = int(pad_rate * ncol1)
    # 1. edge column for an even width, centring shift: all rows of all
    # slices in one launch
    sh = torch.empty((nrow, nslice, ncol1), dtype=torch.float32, device=dev)
    nat.call("atb_shift_rows_ext", t.data_ptr(), t.stride(-2),
             nrow * nslice, ncol, ncol1, float(xshift), sh.data_ptr(),
             ncol1, st)
    # 2. angles
    if angles is not None:
        sh = _angle_rows(sh, angles)
    w = ncol1 + 2 * pad
    window = _window(filter_name, w, dev) if filter_name is not None \
        else None
    mask_r2 = -1.0
    if ratio is not None:
        if ratio == 0.0:
            ratio = min(center, ncol - center) / (0.5 * ncol)
        radius = ratio * (ncol // 2)
        mask_r2 = radius * radius
    dtype = torch.float64 if filter_name is not None else torch.float32
    shape = (ncol, nslice, ncol) if input_3d else (ncol, ncol)
    out = torch.empty(shape, dtype=dtype, device=dev)
    run = _dfi_own if _own_transform(w) else _dfi_wide
    bad = run(sh, out, pad, ncol, pad_mode, apply_log is True, window,
              mask_r2)
    if bad:
        warnings.warn("!!!Applying logarithm is enabled but "
                      "there are values <= 0.0 in the data!!!")
    return out.cpu().numpy() if is_np else out
