"""FP64 NumPy restatement of algotom's vertical-slice reconstruction.

TEST INFRASTRUCTURE ONLY -- imported by tests and the CPU legs of
``bench.py`` as the checker.  Never part of the product path.

Restates, citing algotom 1.6.0 ``algotom/rec/vertrec.py``:

- the vertical back-projectors (``:53-335``): for every angle a_n and
  point (x_j, y_j) of a slice, position p = x cos a + y sin a + center; for
  every detector row i the interpolated sample of projection n at p (inclusive
  bounds [0, width-1], y[d] when ceil(p) == floor(p), edge padding with the
  end samples), summed over n -- here in FP64 throughout;
- the slice geometry ``_get_points_single_line`` (``:338-384``), evaluated
  with the same NumPy expressions (it defines the points);
- the chunked drivers (``:450-1252``): flat/dark correction, ``-log`` with
  values <= 0 set to 1, the ramp filter before (``apply_ramp_filter`` on each
  projection) or after (``|W|`` zero-phase filter of each slice row,
  ``:698-706``) the back-projection, masking, scale pi / (num_proj - 1).
"""
import numpy as np

from . import fbp_oracle as O


def points_single_line(slice_index, alpha, width):
    """``_get_points_single_line`` (vertrec.py:338-384)."""
    if alpha < 0.0 or alpha > 180.0:
        raise ValueError("Angle is out of range [0, 180] (degree)")
    if slice_index < 0 or slice_index > width - 1:
        raise ValueError("Slice index is out of range")
    center = np.ceil(0.5 * (width - 1))
    x_min, x_max = - center, width - center
    angle = np.deg2rad(alpha)
    x0 = y0 = slice_index - center
    if alpha <= 45 or alpha >= 135:
        a = np.tan(angle)
        b = - y0 / np.cos(angle)  # the radians-vs-45 test always holds
        xcr = - a * b / (1 + a ** 2)
        xs = xcr + np.arange(x_min, x_max) * np.cos(angle)
        ys = a * xs + b
    else:
        a = np.cos(angle) / np.sin(angle)
        b = x0 / np.sin(angle)  # the radians-vs-90 test always holds
        ycr = - a * b / (1 + a ** 2)
        ys = ycr + np.arange(x_min, x_max) * np.sin(angle)
        xs = a * ys + b
    return xs, ys


def vertical_back_projection(projections, angles, xs, ys, center,
                             edge_pad=False):
    """FP64 vertical back-projection: projections [depth, height, width],
    points (xs, ys) of one slice -> [height, width]."""
    proj = np.asarray(projections, dtype=np.float64)
    depth, height, width = proj.shape
    xs = np.asarray(xs, dtype=np.float64)[:width]
    ys = np.asarray(ys, dtype=np.float64)[:width]
    w1 = width - 1
    out = np.zeros((height, width))
    for n in range(depth):
        a = float(angles[n])
        p = xs * np.cos(a) + ys * np.sin(a) + center
        inside = (p >= 0) & (p <= w1)
        d = np.floor(np.where(inside, p, 0)).astype(np.int64)
        u = np.ceil(np.where(inside, p, 0)).astype(np.int64)
        f = np.where(inside, p - d, 0.0)
        row = proj[n]
        val = row[:, d] + (row[:, u] - row[:, d]) * f
        val = np.where(inside[None, :], val, 0.0)
        if edge_pad:
            edge = np.where(p < 0, row[:, :1], row[:, w1:w1 + 1])
            val = np.where(inside[None, :], val, edge)
        out += val
    return out


def vertical_back_projection_chunk(projections, angles, x_mat, y_mat,
                                   center, edge_pad=False):
    return np.stack([vertical_back_projection(projections, angles, xs, ys,
                                              center, edge_pad)
                     for xs, ys in zip(x_mat, y_mat)])


def ver_ramp_filter(ver, filter_name, pad, pad_mode):
    """``__apply_ver_ramp_filter`` with ``|W|`` (vertrec.py:684-706)."""
    height, width = ver.shape
    win = np.abs(O.ramp_window_1d(width + 2 * pad, filter_name))
    xp = np.pad(np.asarray(ver, dtype=np.float64), ((0, 0), (pad, pad)),
                mode=pad_mode)
    y = np.fft.ifft(np.fft.ifftshift(np.fft.fftshift(
        np.fft.fft(xp), axes=1) * win[None, :], axes=1))
    return np.real(y)[:, pad:pad + width]


def vertical_reconstruction(projections, x_mat, y_mat, center, angles=None,
                            flat_field=None, dark_field=None,
                            crop=(0, 0, 0, 0), proj_start=0, proj_stop=-1,
                            ramp_filter="after", filter_name="hann",
                            pad=None, pad_mode="edge", apply_log=True,
                            masking=False):
    """FP64 slices [num_slice, height, width] of the points (x_mat, y_mat)
    through the reference's chunked pipeline (chunking does not change the
    FP64 sums)."""
    num_proj0, height0, width0 = projections.shape
    if proj_stop == -1:
        proj_stop = num_proj0
    num_proj = proj_stop - proj_start
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, num_proj))
    top, bot = crop[0], height0 - crop[1]
    left, right = crop[2], width0 - crop[3]
    width = right - left
    proj = np.asarray(projections[proj_start:proj_stop, top:bot, left:right],
                      dtype=np.float64)
    if flat_field is not None or dark_field is not None:
        flat = (np.ones((height0, width0), np.float32) if flat_field is None
                else flat_field)[top:bot, left:right]
        dark = (np.zeros((height0, width0), np.float32) if dark_field is None
                else dark_field)[top:bot, left:right]
        fd = np.float32(flat - dark)
        fd[fd == 0.0] = 1.0
        proj = (proj - dark) / fd
    if apply_log:
        proj = -np.log(np.where(proj <= 0.0, 1.0, proj))
    if pad is None:
        pad = min(int(0.15 * width), 150)
    edge_pad = ramp_filter != "before"
    if ramp_filter == "before":
        proj = np.stack([O.apply_ramp_filter(p, None, filter_name, pad,
                                             pad_mode) for p in proj])
    out = vertical_back_projection_chunk(proj, angles, x_mat, y_mat, center,
                                         edge_pad)
    if ramp_filter == "after":
        out = np.stack([ver_ramp_filter(v, filter_name, pad, pad_mode)
                        for v in out])
    if masking:
        rad = int(min(center, width - center))
        pad_left = (width - 2 * rad) // 2
        m = np.zeros(width)
        m[pad_left:pad_left + 2 * rad] = 1.0
        out = out * m
    return out * np.pi / (num_proj - 1)


def smooth_projections(projections, sigma):
    """``gaussian_filter(projections, (0, sigma, sigma))`` of float32
    projections: the height pass, then the width pass, float32 between them
    (vertrec.py:1348-1349).  Integer projections keep their type, each pass
    truncated toward zero, as scipy's."""
    from .center_oracle import gaussian_filter_rows
    projections = np.asarray(projections)
    dtype = projections.dtype if projections.dtype.kind in "iu" \
        else np.dtype(np.float32)
    out = np.empty(projections.shape, dtype)
    for n, p in enumerate(projections.astype(dtype, copy=False)):
        tmp = gaussian_filter_rows(np.ascontiguousarray(p.T), sigma).T
        out[n] = gaussian_filter_rows(np.ascontiguousarray(tmp), sigma)
    return out


def autocorrelation(img):
    """``mean(max(|ifft(|fft(row)|^2)|, axis=1))`` (vertrec.py:1255-1261),
    FP64."""
    f = np.fft.fft(np.asarray(img, np.float32).astype(np.float64))
    return float(np.mean(np.max(np.abs(np.fft.ifft(np.abs(f) ** 2)),
                                axis=1)))


def find_center_vertical_slice(projections, slice_index, start, stop,
                               step=1.0, metric="entropy", alpha=0.0,
                               angles=None, chunk_size=30,
                               ramp_filter="after", sigma=3, apply_log=True,
                               masking=True, invert_metric=False,
                               metric_function=None, **kwargs):
    """(list_center, list_metric) of ``find_center_vertical_slice``
    (vertrec.py:1264-1383): smoothing, ``-log`` (values <= 0 set to 1),
    one FP64 vertical reconstruction per centre (hann window, edge padding
    of min(0.15 width, 150)), the mask of the smallest centre, and the
    entropy (normalised by the range of the slice at the mean centre, in
    float64 after the "after" ramp filter and float32 otherwise),
    sharpness or autocorrelation metric, or ``metric_function(slice,
    **kwargs)``."""
    from . import center_oracle as C
    if ramp_filter is None:
        ramp_filter = "after"
    list_center = np.arange(start, stop + step, step)
    list_metric = np.zeros_like(list_center)
    num_proj, height, width = projections.shape
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, num_proj))
    proj = np.asarray(projections)
    if proj.dtype.kind not in "iu":
        proj = proj.astype(np.float32)
    if sigma > 0:
        proj = smooth_projections(proj, sigma)
    proj = proj.astype(np.float32).astype(np.float64)
    if apply_log:
        proj = -np.log(np.where(proj <= 0.0, 1.0, proj))
    xs, ys = points_single_line(slice_index, alpha, width)
    pad = min(int(0.15 * width), 150)
    out_dt = np.float64 if ramp_filter == "after" else np.float32

    def recon(center):
        r = vertical_reconstruction(proj, xs[None], ys[None], center,
                                    angles=angles, ramp_filter=ramp_filter,
                                    filter_name="hann", pad=pad,
                                    pad_mode="edge", apply_log=False)[0]
        return r.astype(out_dt)

    mask = None
    if masking:
        rad = int(min(np.min(list_center), width - np.min(list_center)))
        pad_left = (width - 2 * rad) // 2
        mask = np.zeros(width, np.float32)
        mask[pad_left:pad_left + 2 * rad] = 1.0
    if metric_function is None and metric == "entropy":
        first = recon(np.mean(list_center))
        nmin, nmax = first.min(), first.max()
    for i, center in enumerate(list_center):
        r = recon(center)
        if mask is not None:
            r = r * mask.astype(out_dt)
        if metric_function is not None:
            list_metric[i] = metric_function(r, **kwargs)
        elif metric == "entropy":
            if out_dt == np.float32:
                levels = C.normalise_u8(r, nmin, nmax)
            else:
                levels = np.uint8(np.clip((r - nmin) / (nmax - nmin), 0, 1)
                                  * 255)
            list_metric[i] = C.histogram_entropy(levels)
        elif metric == "sharpness":
            list_metric[i] = C.edge_sharpness(r)
        else:
            list_metric[i] = autocorrelation(r)
    if invert_metric:
        list_metric = np.max(list_metric) - list_metric
    return list_center, list_metric
