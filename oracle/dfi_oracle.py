"""FP64 NumPy restatement of algotom's DFI (direct Fourier inversion).

TEST INFRASTRUCTURE ONLY -- imported by tests and the CPU legs of
``bench.py`` as the checker.  Never part of the product path.

Restates ``dfi_reconstruction`` and its helpers (algotom 1.6.0,
``algotom/rec/reconstruction.py:687-907``): pad an even-width sinogram by
one edge column, centre it with a cubic-spline sub-pixel shift, optionally
re-order the angles (``__dfi_handle_angles``), pad the detector axis,
``-log``, transform every row (``fftshift(fft(ifftshift(row)))``), apply the
smoothing window, regrid the polar spectrum onto the Cartesian frequency grid
(``generate_mapping_coordinate`` + ``util.mapping`` = ``map_coordinates``
with quintic splines, ``mode="reflect"``), mask, inverse 2-D transform,
crop and mask.

The scipy.ndimage spline routines it relies on are restated as the
published B-spline algorithms (recursive prefilter with the spline's poles;
boundary start values of the half-sample symmetric extension ("reflect",
also used for "nearest" after 12 edge samples of padding) and of the
whole-sample symmetric one ("mirror", used for "wrap"); samples with the
B-spline weights at clamped / reflected / mirrored taps).
"""
from math import comb

import numpy as np

from . import fbp_oracle as O

POLES = {3: (np.sqrt(3.0) - 2.0,),
         5: (np.sqrt(135.0 / 2.0 - np.sqrt(17745.0 / 4.0)) +
             np.sqrt(105.0 / 4.0) - 13.0 / 2.0,
             np.sqrt(135.0 / 2.0 + np.sqrt(17745.0 / 4.0)) -
             np.sqrt(105.0 / 4.0) - 13.0 / 2.0)}


def _causal_reflect(c, z):
    n, z_i, z_n, c0 = len(c), z, z ** len(c), c[0]
    s = c[0] + z_n * c[n - 1]
    for i in range(1, n):
        s += z_i * (c[i] + z_n * c[n - 1 - i])
        z_i *= z
    return s * (z / (1 - z_n * z_n)) + c0


def _causal_mirror(c, z):
    n, z_i = len(c), z
    z_n1 = z ** (n - 1)
    s = c[0] + z_n1 * c[n - 1]
    for i in range(1, n - 1):
        s += z_i * (c[i] + z_n1 * c[n - 1 - i])
        z_i *= z
    return s / (1 - z_n1 * z_n1)


def spline_filter1d(x, order, boundary):
    """B-spline coefficients along the last axis; ``boundary`` is
    "reflect" (half-sample symmetric) or "mirror" (whole-sample)."""
    c = np.array(x, dtype=np.result_type(x, np.float64), copy=True)
    n = c.shape[-1]
    lam = 1.0
    for z in POLES[order]:
        lam *= (1 - z) * (1 - 1 / z)
    c *= lam
    if n == 1:
        return c
    flat = c.reshape(-1, n)
    for row in flat:
        for z in POLES[order]:
            if boundary == "reflect":
                row[0] = _causal_reflect(row, z)
            else:
                row[0] = _causal_mirror(row, z)
            for i in range(1, n):
                row[i] += z * row[i - 1]
            if boundary == "reflect":
                row[n - 1] = row[n - 1] * z / (z - 1)
            else:
                row[n - 1] = (z * row[n - 2] + row[n - 1]) * z / (z * z - 1)
            for i in range(n - 2, -1, -1):
                row[i] = z * (row[i + 1] - row[i])
    return c


def bspline(u, order):
    """Centred B-spline of ``order`` at ``u``."""
    u = np.abs(u)
    h = (order + 1) / 2.0
    s = 0.0
    for k in range(order + 2):
        s = s + (-1) ** k * comb(order + 1, k) * \
            np.maximum(u + h - k, 0.0) ** order
    return s / float(np.prod(np.arange(1, order + 1)))


def _reflect(i, n):
    p = 2 * n
    r = np.mod(i, p)
    return np.where(r >= n, p - 1 - r, r)


def _mirror(i, n):
    if n == 1:
        return np.zeros_like(i)
    p = 2 * (n - 1)
    r = np.mod(i, p)
    return np.where(r >= n, p - r, r)


def shift_cols_wrap(mat, s):
    """float32 ``scipy.ndimage.shift(mat, (s, 0), mode="wrap")``."""
    mat = np.asarray(mat)
    n = mat.shape[0]
    c = np.moveaxis(spline_filter1d(np.moveaxis(mat.astype(np.float64), 0,
                                                -1), 3, "mirror"), -1, 0)
    cc = np.arange(n, dtype=np.float64) - s
    sz = n - 1
    if sz > 0:
        cc = np.where(cc < 0, cc + sz * (np.floor(-cc / sz) + 1), cc)
        cc = np.where(cc > n - 1, cc - sz * np.floor(cc / sz), cc)
    f = np.floor(cc).astype(np.int64)
    out = np.zeros(mat.shape)
    for m in range(-1, 3):
        w = bspline(cc - (f + m), 3)
        out += w[:, None] * c[_mirror(f + m, n)]
    return out.astype(mat.dtype)


def mapping_coordinates(width_sino, height_sino, width_rec, height_rec):
    """``generate_mapping_coordinate`` (reconstruction.py:687-728)."""
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


def map_coordinates5(img, rows, cols):
    """``map_coordinates(img, [rows, cols], order=5, mode="reflect")``."""
    c = spline_filter1d(img, 5, "reflect")
    c = np.moveaxis(spline_filter1d(np.moveaxis(c, 0, -1), 5, "reflect"),
                    -1, 0)
    h, w = img.shape
    rows = np.asarray(rows, np.float64)
    cols = np.asarray(cols, np.float64)
    fr = np.floor(rows).astype(np.int64)
    fc = np.floor(cols).astype(np.int64)
    out = np.zeros(rows.shape, dtype=c.dtype)
    for a in range(6):
        ia = fr - 2 + a
        wa = bspline(rows - ia, 5)
        for b in range(6):
            ib = fc - 2 + b
            out += wa * bspline(cols - ib, 5) * c[_reflect(ia, h),
                                                   _reflect(ib, w)]
    return out


def handle_angles(sinogram, angles):
    """``__dfi_handle_angles`` (reconstruction.py:731-749)."""
    nrow = sinogram.shape[0]
    t_ang = np.sum(np.abs(np.diff(angles * 180.0 / np.pi)))
    if abs(t_ang - 360) < 10:
        nrow = nrow // 2 + 1
        sinogram = (sinogram[:nrow] + np.fliplr(sinogram[-nrow:])) / 2
    step = np.mean(np.abs(np.diff(angles)))
    b_ang = angles[0] - (angles[0] // (2 * np.pi)) * (2 * np.pi)
    sino_360 = np.vstack((sinogram[: nrow - 1], np.fliplr(sinogram)))
    sinogram = shift_cols_wrap(sino_360, b_ang / step)[:nrow]
    if angles[-1] < angles[0]:
        sinogram = np.flipud(np.fliplr(sinogram))
    return sinogram


def dfi_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       filter_name="hann", pad_rate=0.25, pad_mode="edge",
                       apply_log=True):
    """FP64 DFI of a 2-D sinogram (``reconstruction.py:818-907``)."""
    from .conversion_oracle import shift_rows
    sino = np.asarray(sinogram, dtype=np.float32)
    nrow, ncol = sino.shape
    if ncol % 2 == 0:
        sino = np.pad(sino, ((0, 0), (0, 1)), mode="edge")
    ncol1 = sino.shape[-1]
    xshift = (ncol1 - 1) / 2.0 - center
    pad = int(pad_rate * ncol1)
    sino = shift_rows(sino, xshift)
    if angles is not None:
        sino = handle_angles(sino, np.asarray(angles, np.float64))
    sino = np.pad(sino, ((0, 0), (pad, pad)), mode=pad_mode)
    sino = sino.astype(np.float64)
    if apply_log:
        sino = -np.log(np.where(sino <= 0.0, 1.0, sino))
    nrow, ncol2 = sino.shape
    mask = O.make_circle_mask(ncol2, 1.0)
    r_mat, theta_mat = mapping_coordinates(ncol2, nrow, ncol2, ncol2)
    f = np.fft.fftshift(np.fft.fft(np.fft.ifftshift(sino, axes=1)), axes=1)
    if filter_name is not None:
        f = f * O.make_smoothing_window(filter_name, ncol2)[None, :]
    reg = map_coordinates5(f, theta_mat, r_mat) * mask
    rec = np.real(np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(reg))))
    rec = rec[pad:ncol + pad, pad:ncol + pad]
    if ratio is not None:
        if ratio == 0.0:
            ratio = min(center, ncol - center) / (0.5 * ncol)
        rec = rec * O.make_circle_mask(ncol, ratio)
    return rec


def dfi_reconstruction_scipy(sinogram, center, ratio=1.0, filter_name="hann",
                             pad_rate=0.25, pad_mode="edge"):
    """The same steps (no angle handling, no -log) through scipy.ndimage's
    compiled spline routines and NumPy's FFT, as the reference calls them:
    the timed CPU baseline at full size, where the pure-Python restatement
    above would take minutes."""
    import scipy.ndimage as ndi
    sino = np.asarray(sinogram, dtype=np.float32)
    nrow, ncol = sino.shape
    if ncol % 2 == 0:
        sino = np.pad(sino, ((0, 0), (0, 1)), mode="edge")
    ncol1 = sino.shape[-1]
    pad = int(pad_rate * ncol1)
    sino = ndi.shift(sino, (0, (ncol1 - 1) / 2.0 - center), mode="nearest")
    sino = np.pad(sino, ((0, 0), (pad, pad)), mode=pad_mode)
    nrow, ncol2 = sino.shape
    mask = O.make_circle_mask(ncol2, 1.0)
    r_mat, theta_mat = mapping_coordinates(ncol2, nrow, ncol2, ncol2)
    f = np.fft.fftshift(np.fft.fft(np.fft.ifftshift(sino, axes=1)), axes=1)
    if filter_name is not None:
        f = f * O.make_smoothing_window(filter_name, ncol2)[None, :]
    coords = np.vstack((theta_mat.ravel(), r_mat.ravel()))
    reg = ndi.map_coordinates(f, coords, order=5, mode="reflect").reshape(
        r_mat.shape) * mask
    rec = np.real(np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(reg))))
    rec = rec[pad:ncol + pad, pad:ncol + pad]
    if ratio is not None:
        rec = rec * O.make_circle_mask(ncol, ratio)
    return rec
