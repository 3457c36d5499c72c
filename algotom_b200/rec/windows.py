"""Host-side FP64 construction of the filter constants the kernels consume.

Smoothing windows, ramp windows and circular ramp windows keep algotom's
definitions (``algotom/rec/reconstruction.py:50-115, 496-524``;
``algotom/util/utility.py:131-157, 925-963``), built with the same
``scipy.signal.windows`` / ``scipy.ndimage.map_coordinates`` calls.

:func:`row_filter_spectrum` turns a Fourier-space ramp window of width
``N = ncol + 2 pad`` into what ``atb_filter_rows`` needs: the spectrum of
the periodised real kernel at the transform length ``atb_filter_length``
chooses, ``N`` itself or an embedding length ``M >= N + ncol - 1``.
Derivation: algotom's filter is
``crop(ifftshift(real(ifft(ifftshift(fftshift(fft(x)) W)))))``; the two
spectrum shifts cancel, so with ``H = ifftshift(W)`` the output is the real
circular convolution of the padded row with
``kappa = roll(real(ifft(H)), -(N // 2))``, cropped to ``[pad, pad+ncol)``.
Those outputs use kernel lags ``u`` in ``[pad - N + 1, pad + ncol - 1]``
only, so a length-M circular convolution with ``b[u mod M] = kappa[u mod N]``
on those lags (zero elsewhere) gives the same values at the same
positions.  Taking ``real`` of the inverse transform keeps only the
Hermitian part of ``H``, which this construction inherits automatically.
"""
import math

import numpy as np
import scipy.ndimage as ndi
import scipy.signal.windows as sigwin

WINDOW_NAMES = ("hann", "bartlett", "blackman", "hamming", "nuttall",
                "parzen", "triang")


def make_smoothing_window(filter_name, width):
    """1-D smoothing window; ``None`` or an unknown name gives ones.

    Same windows as ``algotom/rec/reconstruction.py:50-83``.
    """
    if filter_name in WINDOW_NAMES:
        return getattr(sigwin, filter_name)(width)
    return np.ones(width)


def _ramp_kernel(width):
    # k = i - ceil((width-1)/2): 0.25 at 0, 0 at even k, -1/(pi k)^2 at odd k
    k = np.arange(width, dtype=np.float64) - math.ceil((width - 1.0) / 2)
    r = np.zeros(width)
    odd = (np.abs(k) % 2) == 1
    r[odd] = -1.0 / (np.pi * k[odd]) ** 2
    r[k == 0] = 0.25
    return r


def ramp_window_row(width, filter_name=None):
    """``fftshift(fft(ramp)) * window`` (``reconstruction.py:103-110``)."""
    return np.fft.fftshift(np.fft.fft(_ramp_kernel(width))) * \
        make_smoothing_window(filter_name, width)


def make_2d_ramp_window(height, width, filter_name=None):
    """Ramp window tiled to (height, width); ``reconstruction.py:86-115``."""
    return np.tile(ramp_window_row(width, filter_name), (height, 1))


def row_filter_spectrum(window_rows, ncol, pad, m):
    """FP64 spectrum of the periodised kernel for each row of a ramp window.

    ``window_rows``: complex [R, N] Fourier-space window rows in fftshifted
    order (R = 1 for a tiled window).  ``m``: the transform length, N itself
    or at least N + ncol - 1 (``atb_filter_length``).  Returns complex64
    [R, m] already multiplied by 1/m (the kernel's inverse transform is an
    unnormalised forward FFT of the conjugate).
    """
    w = np.atleast_2d(np.asarray(window_rows, dtype=np.complex128))
    n = ncol + 2 * pad
    if w.shape[1] != n:
        raise ValueError("window width %d != ncol + 2*pad = %d"
                         % (w.shape[1], n))
    if m != n and m < n + ncol - 1:
        raise ValueError("transform length %d is neither N = %d nor at "
                         "least N + ncol - 1 = %d" % (m, n, n + ncol - 1))
    h = np.fft.ifftshift(w, axes=1)
    kappa = np.roll(np.real(np.fft.ifft(h, axis=1)), -(n // 2), axis=1)
    if m == n:
        b = kappa
    else:
        lags = np.arange(pad - n + 1, pad + ncol)
        b = np.zeros((w.shape[0], m))
        b[:, lags % m] = kappa[:, lags % n]
    return (np.fft.fft(b, axis=1) / m).astype(np.complex64)


def make_circular_ramp_window(width, filter_name=None):
    """2-D circular ramp window; ``reconstruction.py:496-524``.

    ``|fftshift(fft(ramp))| * window`` swept around the centre: output pixel
    (row, col) of a (w x w) grid, w odd (even widths are built at w + 1 and
    cropped), samples the 1-D profile at the signed radius (negative for
    polar angles below zero, offset by the centre) along columns and at a
    row index proportional to the polar angle, with order-1 interpolation
    and nearest-edge extension, as ``algotom/util/utility.py:925-963`` does.
    """
    prof = np.abs(np.fft.fftshift(np.fft.fft(_ramp_kernel(width)))) * \
        make_smoothing_window(filter_name, width)
    w0 = len(prof)
    w = w0 + 1 if w0 % 2 == 0 else w0
    c = w // 2
    xs = np.flipud(np.arange(w)).astype(np.float64) - c
    ys = np.arange(w).astype(np.float64) - c
    xm, ym = np.meshgrid(xs, ys)
    rad = np.float32(np.clip(np.sqrt(xm ** 2 + ym ** 2), 0, c))
    ang = np.arctan2(ym, xm)
    rad[ang < 0] *= -1
    rad = np.float32(np.clip(rad + c, 0, w - 1))
    ang = np.clip(np.float32(ang * (w - 1.0) / np.pi), 0, w - 1)
    grid = np.tile(prof, (w, 1))
    vals = ndi.map_coordinates(grid, np.vstack((ang.ravel(), rad.ravel())),
                               order=1, mode="nearest")
    return vals.reshape(xm.shape)[:w0, :w0]


def make_circle_mask(width, ratio):
    """Disc mask of radius ratio*(width//2); ``utility.py:160-182``."""
    c = width // 2
    idx = np.arange(width) - c
    r = ratio * c
    return ((idx[None, :] ** 2 + idx[:, None] ** 2) <= r * r
            ).astype(np.float32)
