"""FP64 NumPy restatement of algotom's 360-degree sinogram conversions.

TEST INFRASTRUCTURE ONLY -- imported by tests as the checker.  Never part of
the product path.

Restates, citing algotom 1.6.0 ``algotom/prep/conversion.py``:

- ``make_weight_matrix`` (``:43-73``) and ``stitch_image`` (``:76-144``);
- ``convert_sinogram_360_to_180`` (``:318-364``),
  ``convert_sinogram_180_to_360`` (``:367-392``) and ``extend_sinogram``
  (``:395-454``);
- the sub-pixel ``scipy.ndimage.shift(x, (0, s), mode="nearest")`` they call
  (default spline order 3), as the published algorithm it is: the row is
  padded with 12 copies of each end sample, turned into cubic B-spline
  coefficients by the recursive filter with pole sqrt(3) - 2 (gain
  (1 - z)(1 - 1/z), causal start value of the half-sample symmetric
  extension, anti-causal start value z / (z - 1) c[n-1]), and sampled at
  x - s with the cubic B-spline weights, coefficient indices clamped to the
  padded row.  Along axis 0 the shift is zero, and a cubic spline sampled at
  its knots returns its samples, so rows are independent.
"""
import numpy as np

_Z = np.sqrt(3.0) - 2.0
_NPAD = 12


def spline_coefficients(x):
    """Cubic B-spline coefficients of a 1-D FP64 signal (in a copy)."""
    c = np.asarray(x, dtype=np.float64).copy()
    n, z = len(c), _Z
    c *= (1.0 - z) * (1.0 - 1.0 / z)
    if n == 1:
        return c
    z_i, z_n, c0 = z, z ** n, c[0]
    s = c[0] + z_n * c[n - 1]
    for i in range(1, n):
        s += z_i * (c[i] + z_n * c[n - 1 - i])
        z_i *= z
    c[0] = s * (z / (1.0 - z_n * z_n)) + c0
    for i in range(1, n):
        c[i] += z * c[i - 1]
    c[n - 1] *= z / (z - 1.0)
    for i in range(n - 2, -1, -1):
        c[i] = z * (c[i + 1] - c[i])
    return c


def shift_row(x, s):
    """``scipy.ndimage.shift(x, s, mode="nearest")`` of one row, FP64."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    c = spline_coefficients(np.pad(x, _NPAD, mode="edge"))
    big = len(c)
    cc = (np.arange(n, dtype=np.float64) - s) + _NPAD
    f = np.floor(cc)
    t = cc - f
    i0 = f.astype(np.int64)
    w = ((1 - t) ** 3 / 6.0, (4 - 6 * t * t + 3 * t ** 3) / 6.0,
         (1 + 3 * t + 3 * t * t - 3 * t ** 3) / 6.0, t ** 3 / 6.0)
    out = np.zeros(n)
    for m, wm in zip(range(-1, 3), w):
        out += wm * c[np.clip(i0 + m, 0, big - 1)]
    return out


def shift_rows(mat, s):
    """Float32 result of ``scipy.ndimage.shift(mat, (0, s), mode="nearest")``
    for a float32 2-D array."""
    mat = np.asarray(mat)
    return np.stack([shift_row(r, s) for r in mat]).astype(mat.dtype)


def _overlap_side(cor, ncol):
    if isinstance(cor, tuple):
        return cor
    if cor <= (ncol - 1.0) * 0.5:
        return 2 * cor + 1, 0
    return 2 * (ncol - cor) - 1, 1


def make_weight_matrix(mat1, mat2, overlap, side):
    """``conversion.py:43-73``."""
    overlap = int(np.floor(overlap))
    w1, w2 = np.ones_like(mat1), np.ones_like(mat2)
    down = np.linspace(1.0, 0.0, overlap)
    up = 1.0 - down
    if side == 1:
        w1[:, -overlap:] = np.float32(down)
        w2[:, :overlap] = np.float32(up)
    else:
        w2[:, -overlap:] = np.float32(down)
        w1[:, :overlap] = np.float32(up)
    return w1, w2


def stitch_image(mat1, mat2, overlap, side, wei_mat1=None, wei_mat2=None,
                 norm=True, total_width=None):
    """``conversion.py:76-144`` with FP64 means."""
    nrow1, ncol1 = mat1.shape
    nrow2, ncol2 = mat2.shape
    ov = int(np.round(overlap + 1.0e-3))
    sub = overlap - ov
    if sub != 0.0:
        sgn = 1.0 if side == 1 else -1.0
        mat1 = shift_rows(mat1, sgn * sub)
        mat2 = shift_rows(mat2, -sgn * sub)
    if wei_mat1 is None or wei_mat2 is None:
        wei_mat1, wei_mat2 = make_weight_matrix(mat1, mat2, ov, side)
    tw0 = ncol1 + ncol2 - ov
    if total_width is None or total_width < tw0:
        total_width = tw0
    comb = np.zeros((nrow1, tw0))
    m1, m2 = mat1.astype(np.float64), mat2.astype(np.float64)
    if side == 1:
        if norm:
            m2 = m2 * np.mean(m1[:, -ov:]) / np.mean(m2[:, :ov])
        comb[:, :ncol1] = m1 * wei_mat1
        comb[:, ncol1 - ov:tw0] += m2 * wei_mat2
    else:
        if norm:
            m2 = m2 * np.mean(m1[:, :ov]) / np.mean(m2[:, -ov:])
        comb[:, :ncol2] = m2 * wei_mat2
        comb[:, ncol2 - ov:tw0] += m1 * wei_mat1
    if total_width > tw0:
        comb = np.pad(comb, ((0, 0), (0, total_width - tw0)), mode="edge")
    return comb


def convert_sinogram_360_to_180(sino_360, cor, wei_mat1=None, wei_mat2=None,
                                norm=True, total_width=None):
    """``conversion.py:318-364``."""
    nrow, ncol = sino_360.shape
    n180 = nrow // 2 + 1
    top = sino_360[:n180]
    bot = np.fliplr(sino_360[-n180:])
    overlap, side = _overlap_side(cor, ncol)
    out = stitch_image(top, bot, overlap, side, wei_mat1, wei_mat2, norm,
                       total_width)
    ov = int(np.round(overlap + 1.0e-3))
    return out, ncol - ov / 2.0 - 0.5


def convert_sinogram_180_to_360(sino_180, center):
    """``conversion.py:367-392``."""
    nrow, ncol = sino_180.shape
    sx = (ncol - 1.0) / 2.0 - center
    flip = shift_rows(np.fliplr(shift_rows(sino_180, sx)), -sx)
    return np.vstack((sino_180, flip[1:]))


def extend_sinogram(sino_360, cor, apply_log=True):
    """``conversion.py:395-454`` in FP64 after the float32 input."""
    s = np.asarray(sino_360, dtype=np.float64)
    if apply_log:
        s = -np.log(s)
    nrow, ncol = s.shape
    overlap, side = _overlap_side(cor, ncol)
    ov = int(np.round(overlap + 1.0e-3))
    sub = overlap - ov
    if side == 1:
        if sub != 0.0:
            s = np.stack([shift_row(r, sub) for r in s])
        s[:, -ov:] *= np.linspace(1.0, 0.0, ov)[None, :]
        s = np.pad(s, ((0, 0), (0, ncol - ov)), mode="edge")
    else:
        if sub != 0.0:
            s = np.stack([shift_row(r, -sub) for r in s])
        s[:, :ov] *= np.linspace(0.0, 1.0, ov)[None, :]
        s = np.pad(s, ((0, 0), (ncol - ov, 0)), mode="edge")
    return 2 * s, ncol - ov / 2.0 - 0.5
