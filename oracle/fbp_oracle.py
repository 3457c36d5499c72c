"""FP64 NumPy restatement of algotom's FBP / BPF hot path.

TEST INFRASTRUCTURE ONLY -- imported by tests, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py`` as the checker.  Never part of the product path.

Each function cites the reference (algotom 1.6.0) file:line it restates.  The
arithmetic is FP64 throughout.  Following the reference, angles and the centre
are rounded to float32 first (``algotom/rec/reconstruction.py:452-457`` passes
``np.float32(angles)`` / ``np.float32(center)`` to every back-projector), and
the trigonometry is then evaluated in FP64 on those float32 values.

Third-party arithmetic used exactly where the reference uses it:
``scipy.signal.windows`` for the smoothing windows
(``reconstruction.py:68-82``), ``numpy.pad`` for the padding modes
(``reconstruction.py:146,556``) and ``scipy.ndimage.map_coordinates`` for the
2-D circular window (``utility.py:156``).  The FFT filter itself is restated as
the real circular convolution it is (see :func:`apply_ramp_filter`).
"""
import math

import numpy as np
import scipy.ndimage as ndi
import scipy.signal.windows as sigwin

WINDOW_NAMES = ("hann", "bartlett", "blackman", "hamming", "nuttall",
                "parzen", "triang")


# --------------------------------------------------------------------------
# Windows and ramp kernels
# --------------------------------------------------------------------------
def make_smoothing_window(filter_name, width):
    """Symmetric smoothing window; unknown names or ``None`` give ones.

    Restates ``algotom/rec/reconstruction.py:50-83``.
    """
    if filter_name in WINDOW_NAMES:
        return getattr(sigwin, filter_name)(width)
    return np.ones(width)


def ramp_spatial(width):
    """Spatial ramp kernel sampled at k = i - ceil((width-1)/2).

    0.25 at k = 0, 0 at even k, -1/(pi k)^2 at odd k.  Restates
    ``algotom/rec/reconstruction.py:103-108``.
    """
    k = np.arange(width, dtype=np.float64) - math.ceil((width - 1.0) / 2)
    r = np.zeros(width)
    odd = (np.abs(k) % 2) == 1
    r[odd] = -1.0 / (k[odd] * np.pi) ** 2
    r[k == 0] = 0.25
    return r


def ramp_window_1d(width, filter_name=None):
    """One row of the Fourier-space ramp window, in fftshifted order.

    ``fftshift(fft(ramp)) * window`` (``reconstruction.py:109-110``).
    """
    r = ramp_spatial(width)
    return np.fft.fftshift(np.fft.fft(r)) * make_smoothing_window(filter_name,
                                                                  width)


def make_2d_ramp_window(height, width, filter_name=None):
    """The 1-D window tiled to (height, width); ``reconstruction.py:86-115``."""
    return np.tile(ramp_window_1d(width, filter_name), (height, 1))


def _pad_rows(sino, pad, pad_mode):
    """``np.pad`` along the detector axis, as ``reconstruction.py:146``."""
    return np.pad(np.asarray(sino, dtype=np.float64), ((0, 0), (pad, pad)),
                  mode=pad_mode)


def apply_ramp_filter(sinogram, ramp_win=None, filter_name=None, pad=None,
                      pad_mode="edge"):
    """FP64 ramp filter of a 2-D sinogram.

    Restates ``algotom/rec/reconstruction.py:118-153``.  The reference computes
    ``ifftshift(ifft(ifftshift(fftshift(fft(x)) * W)))`` and keeps the real
    part; shifting the spectrum back and forth cancels, so with
    ``H = ifftshift(W)`` this is ``roll(real(ifft(fft(x) * H)), -(N // 2))``:
    a real circular convolution of the padded row, rolled and cropped.  When
    ``H`` is not Hermitian (even N) only its Hermitian part survives ``real``.
    """
    sinogram = np.asarray(sinogram)
    nrow, ncol = sinogram.shape
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    xp = _pad_rows(sinogram, pad, pad_mode)
    n = ncol + 2 * pad
    if (ramp_win is None) or (np.shape(ramp_win) != xp.shape):
        ramp_win = make_2d_ramp_window(nrow, n, filter_name)
    h = np.fft.ifftshift(np.asarray(ramp_win, dtype=np.complex128), axes=1)
    y = np.real(np.fft.ifft(np.fft.fft(xp, axis=1) * h, axis=1))
    y = np.roll(y, -(n // 2), axis=1)
    return np.ascontiguousarray(y[:, pad:pad + ncol])


def filter_kernel_spatial(width, filter_name=None):
    """Real periodic kernel kappa with filtered[n] = sum_k x[k] kappa[n-k].

    ``kappa = roll(real(ifft(ifftshift(W))), -(N // 2))`` for the tiled
    window of ``make_2d_ramp_window`` (``reconstruction.py:86-115``); this is
    the convolution form of :func:`apply_ramp_filter` (indices mod N) for a
    row-invariant window.
    """
    h = np.fft.ifftshift(ramp_window_1d(width, filter_name))
    kappa = np.real(np.fft.ifft(h))
    return np.roll(kappa, -(width // 2))


# --------------------------------------------------------------------------
# Back-projection
# --------------------------------------------------------------------------
def back_projection(sinogram, angles, center, edge_pad=False,
                    round_inputs=True):
    """FP64 linear-interpolation back-projection of one sinogram.

    Restates ``back_projection_cpu`` (``reconstruction.py:307-359``) and the
    GPU kernel ``reconstruction.py:156-190``: pixel (y, x) reads detector
    position ``p = (x-ic) cos(-t) + (y-ic) sin(-t) + center`` with
    ``ic = (ncol-1)/2``.  If ``0 <= p <= ncol-1`` it adds
    ``s[d] + (s[u]-s[d]) (p-d)`` with ``d = floor(p)``, ``u = ceil(p)`` (just
    ``s[d]`` when ``u == d``); otherwise it adds ``s[0]`` (``p < 0``) or
    ``s[ncol-1]`` when ``edge_pad``, else nothing.  Angles and centre are
    rounded to float32 first, as the reference does before every call
    (``round_inputs=False`` keeps them exact, for derivative checks).
    """
    sino = np.asarray(sinogram, dtype=np.float64)
    nrow, ncol = sino.shape
    if round_inputs:
        ang = np.float32(np.asarray(angles)).astype(np.float64)
        cen = float(np.float32(center))
    else:
        ang = np.asarray(angles, dtype=np.float64)
        cen = float(center)
    ic = 0.5 * (ncol - 1)
    xc = np.arange(ncol, dtype=np.float64) - ic
    out = np.zeros((ncol, ncol))
    for i in range(nrow):
        c = math.cos(-ang[i])
        s = math.sin(-ang[i])
        p = xc[None, :] * c + xc[:, None] * s + cen
        inside = (p >= 0.0) & (p <= ncol - 1)
        pc = np.where(inside, p, 0.0)
        d = np.floor(pc).astype(np.int64)
        u = np.ceil(pc).astype(np.int64)
        row = sino[i]
        val = row[d] + (row[u] - row[d]) * (pc - d)
        val = np.where(inside, val, 0.0)
        if edge_pad:
            val = np.where(p < 0.0, row[0], val)
            val = np.where(p > ncol - 1, row[ncol - 1], val)
        out += val
    return out


def forward_projection(image, angles, center):
    """FP64 adjoint of :func:`back_projection` (no edge padding).

    Scatters each pixel with position ``p`` in ``[0, ncol-1]`` onto bins
    ``floor(p)`` and ``floor(p)+1`` with weights ``1-f`` and ``f`` -- the
    transpose of the reference back-projector's interpolation
    (``reconstruction.py:307-359``).  Angles and centre are used as given
    (no float32 rounding), as for a differentiable model.
    """
    img = np.asarray(image, dtype=np.float64)
    ncol = img.shape[0]
    ang = np.asarray(angles, dtype=np.float64)
    ic = 0.5 * (ncol - 1)
    xc = np.arange(ncol, dtype=np.float64) - ic
    out = np.zeros((len(ang), ncol))
    for i, a in enumerate(ang):
        p = xc[None, :] * math.cos(-a) + xc[:, None] * math.sin(-a) + center
        ok = (p >= 0.0) & (p <= ncol - 1)
        pc = p[ok]
        v = img[ok]
        d = np.floor(pc).astype(np.int64)
        f = pc - d
        np.add.at(out[i], d, (1.0 - f) * v)
        hi = d + 1 <= ncol - 1
        np.add.at(out[i], d[hi] + 1, (f * v)[hi])
    return out


def back_projection_stack(sinograms, angles, center, edge_pad=False):
    """[nrow, nslice, ncol] -> [ncol, nslice, ncol]; ``reconstruction.py:229-304``."""
    nrow, nslice, ncol = sinograms.shape
    out = np.zeros((ncol, nslice, ncol))
    for k in range(nslice):
        out[:, k, :] = back_projection(sinograms[:, k, :], angles, center,
                                       edge_pad)
    return out


# --------------------------------------------------------------------------
# Masks and the BPF 2-D filter
# --------------------------------------------------------------------------
def make_circle_mask(width, ratio):
    """Disc of radius ratio*(width//2) on an integer grid centred at width//2.

    Restates ``algotom/util/utility.py:160-182``.
    """
    c = width // 2
    idx = np.arange(width) - c
    r2 = (ratio * c) ** 2
    return ((idx[None, :] ** 2 + idx[:, None] ** 2) <= r2).astype(np.float32)


def transform_1d_window_to_2d(win_1d, order=1, mode="nearest"):
    """Polar -> Cartesian map of a 1-D window; ``utility.py:925-963``.

    Output pixel (row, col) samples the 1-D window at signed radius
    ``r + c`` (the sign taken from the polar angle) and at a polar row index
    proportional to the angle, through ``map_coordinates``.  Odd sizes are
    built directly, even sizes at width+1 and cropped.
    """
    w0 = len(win_1d)
    w = w0 + 1 if w0 % 2 == 0 else w0
    c = w // 2
    xs = np.flipud(np.arange(w)).astype(np.float64) - c
    ys = np.arange(w).astype(np.float64) - c
    xm, ym = np.meshgrid(xs, ys)
    r = np.float32(np.clip(np.sqrt(xm ** 2 + ym ** 2), 0, c))
    th = np.arctan2(ym, xm)
    r[th < 0] *= -1
    r = np.float32(np.clip(r + c, 0, w - 1))
    th = np.clip(np.float32(th * (w - 1.0) / np.pi), 0, w - 1)
    tiled = np.tile(np.asarray(win_1d), (w, 1))
    coords = np.vstack((th.ravel(), r.ravel()))
    out = ndi.map_coordinates(tiled, coords, order=order, mode=mode)
    return out.reshape(xm.shape)[:w0, :w0]


def make_circular_ramp_window(width, filter_name=None):
    """2-D circular ramp window; ``reconstruction.py:496-524``."""
    r = ramp_spatial(width)
    ramp_1d = np.abs(np.fft.fftshift(np.fft.fft(r))) * \
        make_smoothing_window(filter_name, width)
    return transform_1d_window_to_2d(ramp_1d, order=1, mode="nearest")


def apply_circular_ramp_filter(rec_img, ramp_win=None, filter_name=None,
                               pad=None, pad_mode="edge"):
    """FP64 2-D circular ramp filter; ``reconstruction.py:527-560``.

    ``real(ifft2(fft2(pad(x)) * ifftshift(W2)))`` cropped back to the input.
    """
    ncol = rec_img.shape[0]
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    xp = np.pad(np.asarray(rec_img, dtype=np.float64), pad, mode=pad_mode)
    if (ramp_win is None) or (np.shape(ramp_win) != xp.shape):
        ramp_win = make_circular_ramp_window(ncol + 2 * pad, filter_name)
    h = np.fft.ifftshift(np.asarray(ramp_win))
    y = np.real(np.fft.ifft2(np.fft.fft2(xp) * h))
    return y[pad:pad + ncol, pad:pad + ncol]


# --------------------------------------------------------------------------
# Drivers
# --------------------------------------------------------------------------
def _prepare(sinogram, center, angles, apply_log):
    sino = np.array(sinogram, dtype=np.float64, copy=True)
    if sino.ndim == 3:
        nrow, nslice, ncol = sino.shape
    else:
        nrow, ncol = sino.shape
        nslice = 1
    if center < 0 or center >= ncol:
        raise ValueError("Center is out of the range [0, {}]".format(ncol - 1))
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, nrow))
    elif len(angles) != nrow:
        raise ValueError("Number of angles differs from sinogram rows")
    if apply_log:
        sino[sino <= 0.0] = 1.0
        sino = -np.log(sino)
    return sino, nrow, nslice, ncol, angles


def _mask(ncol, center, ratio):
    if ratio is None:
        return None
    if ratio == 0.0:
        ratio = min(center, ncol - center) / (0.5 * ncol)
    return make_circle_mask(ncol, ratio).astype(np.float64)


def fbp_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       ramp_win=None, filter_name="hann", pad=None,
                       pad_mode="edge", apply_log=True):
    """FP64 FBP of a 2-D or 3-D sinogram; ``reconstruction.py:362-493``.

    -log (values <= 0 read as 1), ramp filter per slice, back-projection
    without edge padding, circle mask, scale pi/(nrow-1).  3-D input is
    [nrow, nslice, ncol] and gives [ncol, nslice, ncol].
    """
    sino, nrow, nslice, ncol, angles = _prepare(sinogram, center, angles,
                                                apply_log)
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    mask = _mask(ncol, center, ratio)
    scale = np.pi / (nrow - 1)
    if sino.ndim == 2:
        f = apply_ramp_filter(sino, ramp_win, filter_name, pad, pad_mode)
        rec = back_projection(f, angles, center)
        if mask is not None:
            rec = rec * mask
        return rec * scale
    rec = np.zeros((ncol, nslice, ncol))
    for k in range(nslice):
        f = apply_ramp_filter(sino[:, k, :], ramp_win, filter_name, pad,
                              pad_mode)
        r = back_projection(f, angles, center)
        rec[:, k, :] = r if mask is None else r * mask
    return rec * scale


def bpf_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       ramp_win=None, filter_name="hann", pad=None,
                       pad_mode="edge", apply_log=True):
    """FP64 BPF; ``reconstruction.py:563-684``.

    -log, back-projection of the unfiltered sinogram WITH edge padding, 2-D
    circular ramp filter per slice, circle mask, scale pi/(nrow-1).
    """
    sino, nrow, nslice, ncol, angles = _prepare(sinogram, center, angles,
                                                apply_log)
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    mask = _mask(ncol, center, ratio)
    scale = np.pi / (nrow - 1)
    if ramp_win is None:
        ramp_win = make_circular_ramp_window(ncol + 2 * pad, filter_name)
    if sino.ndim == 2:
        rec = back_projection(sino, angles, center, edge_pad=True)
        rec = apply_circular_ramp_filter(rec, ramp_win, pad=pad,
                                         pad_mode=pad_mode)
        if mask is not None:
            rec = rec * mask
        return rec * scale
    rec = np.zeros((ncol, nslice, ncol))
    for k in range(nslice):
        r = back_projection(sino[:, k, :], angles, center, edge_pad=True)
        r = apply_circular_ramp_filter(r, ramp_win, filter_name, pad,
                                       pad_mode)
        rec[:, k, :] = r if mask is None else r * mask
    return rec * scale


def rel_l2(a, b):
    """Relative L2 error ||a-b|| / ||b|| in FP64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
