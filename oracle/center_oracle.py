"""FP64 NumPy restatement of algotom's centre search by slice metrics.

TEST INFRASTRUCTURE ONLY -- imported by tests and the CPU legs of
``bench.py`` as the checker.  Never part of the product path.

Restates, citing algotom 1.6.0:

- ``_find_center_based_slice_metric`` (``algotom/rec/reconstruction.py:
  1254-1346``): optional Gaussian smoothing of the sinogram along the
  detector, ``-log``, the normalisation range of the reconstruction at the
  mean candidate (entropy), then a metric per candidate centre and the
  argmin;
- ``find_center_based_slice_metric`` (``:1349-1458``): a coarse pass on a
  linearly zoomed sinogram at unit steps, then a fine pass at ``step``;
- the two metrics, ``__calculate_histogram_entropy`` (``:1212-1221``) and
  ``__calculate_edge_sharpness`` (``:1224-1229``), and the normalisation of
  ``__get_slice_metric`` (``:1232-1251``);
- the two scipy.ndimage pre-steps the reference calls, as the published
  algorithms they are: ``gaussian_filter1d`` (sampled Gaussian normalised to
  unit sum, radius ``int(4 sigma + 0.5)``, symmetric correlation evaluated
  as ``x[i] w0 + sum_j (x[i+j] + x[i-j]) w_j`` in FP64 with half-sample
  symmetric ("reflect") extension, cast to float32) and ``zoom`` with
  ``order=1, mode="nearest"`` (output size ``round(n z)``, sample k at input
  coordinate ``k (n-1)/(m-1)``, bilinear weights, FP64, cast to float32).

Reconstructions use :mod:`oracle.fbp_oracle`.
"""
import numpy as np

from . import fbp_oracle as O


# --------------------------------------------------------------------------
# pre-steps
# --------------------------------------------------------------------------
def gaussian_weights(sigma, truncate=4.0):
    """Half kernel w[0..r] of the unit-sum sampled Gaussian."""
    sigma = float(sigma)
    r = int(truncate * sigma + 0.5)
    x = np.arange(-r, r + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    phi = phi / phi.sum()
    return phi[r:].copy()


def _reflect_index(i, n):
    """Half-sample symmetric extension: ... b a | a b c d | d c ..."""
    period = 2 * n
    i = np.mod(i, period)
    return np.where(i >= n, period - 1 - i, i)


def gaussian_filter_rows(x, sigma):
    """``scipy.ndimage.gaussian_filter1d(x, sigma, axis=1)`` of 2-D float32,
    or of an integer array: then the result has the input's integer type,
    truncated toward zero (the C conversion scipy's correlate1d stores)."""
    dtype = np.asarray(x).dtype
    x = np.asarray(x, dtype=np.float32).astype(np.float64)
    w = gaussian_weights(sigma)
    n = x.shape[1]
    idx = np.arange(n)
    acc = x * w[0]
    for j in range(1, len(w)):
        acc = acc + (x[:, _reflect_index(idx + j, n)] +
                     x[:, _reflect_index(idx - j, n)]) * w[j]
    if dtype.kind in "iu":
        return np.trunc(acc).astype(dtype)
    return acc.astype(np.float32)


def zoom_shape(shape, zoom):
    """Output shape of scipy's zoom (Python's round, half to even)."""
    return tuple(int(round(s * zoom)) for s in shape)


def _zoom_axis(n_in, n_out):
    """Left index, right index and right weight of each output sample."""
    step = (n_in - 1) / (n_out - 1) if n_out > 1 else 1.0
    c = np.arange(n_out, dtype=np.float64) * step
    c = np.clip(c, 0.0, n_in - 1)  # "nearest"
    i0 = np.floor(c).astype(np.int64)
    t = c - i0
    i1 = np.minimum(i0 + 1, n_in - 1)
    return i0, i1, t


def zoom_linear(x, zoom):
    """``scipy.ndimage.zoom(x, zoom, order=1, mode="nearest")`` of 2-D float32."""
    x = np.asarray(x, dtype=np.float32).astype(np.float64)
    m0, m1 = zoom_shape(x.shape, zoom)
    r0, r1, tr = _zoom_axis(x.shape[0], m0)
    c0, c1, tc = _zoom_axis(x.shape[1], m1)
    wr0, wr1 = (1.0 - tr)[:, None], tr[:, None]
    wc0, wc1 = (1.0 - tc)[None, :], tc[None, :]
    out = (x[r0][:, c0] * wr0) * wc0
    out = out + (x[r0][:, c1] * wr0) * wc1
    out = out + (x[r1][:, c0] * wr1) * wc0
    out = out + (x[r1][:, c1] * wr1) * wc1
    return out.astype(np.float32)


# --------------------------------------------------------------------------
# metrics
# --------------------------------------------------------------------------
def normalise_u8(img, nmin, nmax):
    """uint8 levels of ``clip((img - nmin) / (nmax - nmin), 0, 1) * 255``
    in float32 arithmetic (``reconstruction.py:1243-1245``, ``:1216``)."""
    img = np.asarray(img, dtype=np.float32)
    nmin, nmax = np.float32(nmin), np.float32(nmax)
    r = np.clip((img - nmin) / (nmax - nmin), np.float32(0), np.float32(1))
    return (r * np.float32(255)).astype(np.uint8)


def histogram_entropy(levels):
    """``-sum(h log2 h)`` of the 7-wide box sums of ``1 + histogram``."""
    counts = np.bincount(np.asarray(levels).ravel(), minlength=256)
    h = 1.0 + counts.astype(np.float64)
    s = np.array([h[i:i + 7].sum() for i in range(256 - 6)])
    return float(-np.sum(s * np.log2(s)))


def edge_sharpness(img):
    """Mean float32 gradient magnitude (``np.gradient`` stencils)."""
    f = np.asarray(img, dtype=np.float32)
    if min(f.shape) < 2:
        raise ValueError("Shape of array too small to calculate a numerical "
                         "gradient, at least (edge_order + 1) elements are "
                         "required.")
    def grad(a, axis):
        a = np.moveaxis(a, axis, 0)
        g = np.empty_like(a)
        g[1:-1] = (a[2:] - a[:-2]) / np.float32(2.0)
        g[0] = a[1] - a[0]
        g[-1] = a[-1] - a[-2]
        return np.moveaxis(g, 0, axis)
    gy, gx = grad(f, 0), grad(f, 1)
    mag = np.sqrt(gy * gy + gx * gx)
    return float(np.sum(mag.astype(np.float64)) / mag.size)


# --------------------------------------------------------------------------
# drivers
# --------------------------------------------------------------------------
def _reconstruct(sino, center, method, angles, ratio, filter_name):
    fn = {"fbp": O.fbp_reconstruction, "bpf": O.bpf_reconstruction}[method]
    return np.asarray(fn(sino, center, angles=angles, ratio=ratio,
                         filter_name=filter_name, apply_log=False),
                      dtype=np.float32)


def slice_metrics(sinogram, start, stop, step=1, metric="entropy",
                  method="fbp", angles=None, ratio=1.0, filter_name="hann",
                  apply_log=True, sigma=2, invert_metric=False,
                  metric_function=None, **kwargs):
    """(centres, metrics) of ``_find_center_based_slice_metric``."""
    centers = np.arange(start, stop, step)
    if len(centers) == 0:
        raise ValueError("Invalid searching parameters: (start, stop, step)="
                         "{}!!!".format((start, stop, step)))
    sino = np.asarray(sinogram)
    if sino.dtype.kind not in "iu":
        sino = sino.astype(np.float32)
    if sigma > 0:
        sino = gaussian_filter_rows(sino, sigma)
    sino = sino.astype(np.float32)
    if apply_log:
        sino = np.where(sino <= 0.0, np.float32(1.0), sino)
        sino = (-np.log(sino.astype(np.float64))).astype(np.float32)
    nmin = nmax = None
    if metric_function is None and metric == "entropy":
        r = _reconstruct(sino, np.mean(centers), method, angles, ratio,
                         filter_name)
        nmin, nmax = np.min(r), np.max(r)
        if nmin == nmax:
            raise ValueError("Empty image!!!")
    out = np.ones(len(centers))
    for i, c in enumerate(centers):
        r = _reconstruct(sino, c, method, angles, ratio, filter_name)
        if metric_function is not None:
            out[i] = metric_function(r, **kwargs)
        elif metric == "entropy":
            out[i] = histogram_entropy(normalise_u8(r, nmin, nmax))
        else:
            out[i] = edge_sharpness(r)
    if invert_metric:
        out = np.max(out) - out
    return centers, out


def find_center(sinogram, start, stop, step=0.5, metric="entropy", radius=2,
                zoom=1.0, method="fbp", angles=None, ratio=1.0,
                filter_name="hann", apply_log=True, sigma=2,
                invert_metric=False, metric_function=None, **kwargs):
    """Two-pass search of ``find_center_based_slice_metric``."""
    import scipy.ndimage as ndi
    zoom = float(np.clip(zoom, 0.01, 1.0))
    kw = dict(metric=metric, method=method, ratio=ratio,
              filter_name=filter_name, apply_log=apply_log, sigma=sigma,
              invert_metric=invert_metric, metric_function=metric_function,
              **kwargs)
    sino_zoom, angles_zoom = np.asarray(sinogram, dtype=np.float32), angles
    if zoom < 1.0:
        sino_zoom = zoom_linear(sinogram, zoom)
        start, stop = start * zoom, stop * zoom
        if angles is not None:
            # the angle table is host setup: scipy's own 1-D zoom
            angles_zoom = ndi.zoom(np.tile(angles, (1, 1)), (1.0, zoom))[0]
    if stop > start:
        cs, ms = slice_metrics(sino_zoom, start, stop + 1, 1.0,
                               angles=angles_zoom, **kw)
        coarse = cs[np.argmin(ms)] / zoom
    else:
        coarse = start / zoom
    if radius != 0.0:
        radius = max(radius, step + 1.0 / zoom)
        cs, ms = slice_metrics(sinogram, coarse - radius,
                               coarse + radius + step, step, angles=angles,
                               **kw)
        return cs[np.argmin(ms)]
    return coarse
