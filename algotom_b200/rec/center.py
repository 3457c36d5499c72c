"""Centre-of-rotation search by slice metrics on the device.

Drop-in for ``find_center_based_slice_metric`` and
``_find_center_based_slice_metric`` of ``algotom/rec/reconstruction.py``
(algotom 1.6.0, ``:1254-1458``) for the FBP and BPF methods: same names,
signatures, defaults, errors, warnings and results.

The reference reconstructs the slice once per candidate centre, each time
filtering the sinogram again, and evaluates the metric on the host.  Here
the ramp filter (independent of the centre) runs once; the candidates are
then back-projected together: candidates whose float32 centres lie a whole
number of pixels apart share a 4-centre CTA (``atb_backproject_centers``,
one launch per residue class of the progression), others go to ONE
persistent batched launch whose work items share the filtered sinogram and
differ only in their centre (``atb_backproject_batch``).  The metric of
every candidate image is computed on the device (``atb_slice_metric``).  The pre-steps -- Gaussian
smoothing along the detector and the linear zoom of the coarse pass -- are
device kernels with scipy's float32 results (``atb_gaussian_rows``,
``atb_zoom_linear``).  Only the per-candidate metric values (8 bytes each)
come back to the host; a custom ``metric_function`` gets each
reconstruction as a NumPy array, as in the reference.
"""
import ctypes

import numpy as np
import torch

from .. import _native as nat
from . import reconstruction as R

# device bytes of candidate reconstructions held at once
_CHUNK_BYTES = 8 << 30


# --------------------------------------------------------------------------
# device steps
# --------------------------------------------------------------------------
def _gaussian_weights(sigma, truncate=4.0):
    """Half kernel w[0..r] of scipy's unit-sum sampled Gaussian."""
    sigma = float(sigma)
    r = int(truncate * sigma + 0.5)
    x = np.arange(-r, r + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    phi = phi / phi.sum()
    return np.ascontiguousarray(phi[r:])


def _integer_input(x):
    """True when ``x`` (array, tensor or dataset) holds integers: scipy's
    filters then store their output in that integer type, truncated toward
    zero."""
    dt = getattr(x, "dtype", None)
    if isinstance(dt, torch.dtype):
        return not (dt.is_floating_point or dt.is_complex or
                    dt == torch.bool)
    if dt is None:
        dt = np.asarray(x).dtype
    return np.dtype(dt).kind in "iu"


def gaussian_filter_rows(x, sigma, to_int=False):
    """``scipy.ndimage.gaussian_filter1d(x, sigma, axis=1)`` of a 2-D float32
    CUDA tensor (mode "reflect"); returns a new tensor.  ``to_int``: the
    values are integer counts and the results are truncated toward zero, as
    scipy's for an integer array."""
    w = _gaussian_weights(sigma)
    wd = torch.from_numpy(w).to(x.device)
    out = torch.empty(x.shape, dtype=torch.float32, device=x.device)
    nat.call("atb_gaussian_rows", x.data_ptr(), x.stride(0), x.shape[0],
             x.shape[1], wd.data_ptr(), len(w) - 1, out.data_ptr(),
             out.stride(0), int(bool(to_int)), R._stream_ptr(x.device))
    return out


def zoom_image(x, zoom):
    """``scipy.ndimage.zoom(x, zoom, order=1, mode="nearest")`` of a 2-D
    float32 CUDA tensor."""
    rows, cols = (int(round(s * float(zoom))) for s in x.shape)
    out = torch.empty((rows, cols), dtype=torch.float32, device=x.device)
    nat.call("atb_zoom_linear", x.data_ptr(), x.stride(0), x.shape[0],
             x.shape[1], out.data_ptr(), out.stride(0), rows, cols,
             R._stream_ptr(x.device))
    return out


def image_range(img):
    """(min, max) of a 2-D float32 CUDA tensor as NumPy float32 scalars."""
    work = torch.empty(3, dtype=torch.int32, device=img.device)
    out = torch.empty(2, dtype=torch.float32, device=img.device)
    nat.call("atb_image_range", img.data_ptr(), img.stride(0), img.shape[0],
             img.shape[1], work.data_ptr(), out.data_ptr(),
             R._stream_ptr(img.device))
    lo, hi = out.cpu().numpy()
    return np.float32(lo), np.float32(hi)


def slice_metrics(imgs, metric="entropy", nmin=0.0, nmax=1.0):
    """Metric of every image of a [n, rows, cols] float32 CUDA tensor.

    ``"entropy"``: histogram entropy after normalising by (nmin, nmax);
    ``"sharpness"``: mean gradient magnitude.  Returns float64 [n].
    """
    code = nat.METRICS[metric]
    n, rows, cols = imgs.shape
    if imgs.stride(2) != 1:
        imgs = imgs.contiguous()
    nbytes = nat.call("atb_slice_metric_workspace", n, rows, cols, code)
    work = torch.empty(max(int(nbytes), 8), dtype=torch.uint8,
                       device=imgs.device)
    out = torch.empty(n, dtype=torch.float64, device=imgs.device)
    nat.call("atb_slice_metric", imgs.data_ptr(), imgs.stride(0),
             imgs.stride(1), n, rows, cols, code, float(np.float32(nmin)),
             float(np.float32(nmax)), work.data_ptr(), work.numel(),
             out.data_ptr(), R._stream_ptr(imgs.device))
    return out.cpu().numpy()


def _backproject_items(items, device, variant):
    """One persistent batched back-projection of ``nat.BpItem`` s."""
    n = len(items)
    arr = (nat.BpItem * n)(*items)
    nunits = nat.call("atb_bp_batch_plan", ctypes.addressof(arr), n, None, 0,
                      variant)
    units = (ctypes.c_int * nunits)()
    nat.call("atb_bp_batch_plan", ctypes.addressof(arr), n,
             ctypes.addressof(units), nunits, variant)
    items_dev = torch.frombuffer(bytearray(bytes(arr)),
                                 dtype=torch.uint8).to(device)
    units_dev = torch.frombuffer(bytearray(bytes(units)),
                                 dtype=torch.int32).to(device)
    counter = torch.zeros(2, dtype=torch.int32, device=device)
    nat.call("atb_backproject_batch", items_dev.data_ptr(), n,
             units_dev.data_ptr(), nunits, counter.data_ptr(), 0, variant,
             R._stream_ptr(device))
    # the caching allocator keeps these until the stream has used them
    return items_dev, units_dev, counter


def _centre_groups(centers, max_classes=16, max_spacing=56):
    """Split candidate centres into progressions whose float32 values differ
    by whole pixels: ``[(r, R, c0, spacing, count)]`` where candidates
    ``r, r + R, r + 2R, ...`` sit at exactly ``c0 + m * spacing``.  None
    when no ``R <= max_classes`` splits them so (e.g. irregular centres).
    Such candidates share one back-projection (``atb_backproject_centers``):
    a centre one pixel further reads the same positions one detector bin
    further."""
    c = np.float32(np.asarray(centers, dtype=np.float64)).astype(np.float64)
    n = len(c)
    if n < 2:
        return None
    for nclass in range(1, min(max_classes, n) + 1):
        groups = []
        for r in range(nclass):
            cls = c[r::nclass]
            d = np.diff(cls)
            if len(d) == 0:
                groups.append((r, nclass, float(cls[0]), 1, 1))
                continue
            g = d[0]
            if not (g == np.round(g) and 1 <= g <= max_spacing and
                    np.all(d == g)):
                break
            groups.append((r, nclass, float(cls[0]), int(g), len(cls)))
        else:
            return groups
    return None


class _Source:
    """The sinogram of one search, prepared once for every candidate: the
    ramp-filtered rows for FBP, the -log rows for BPF."""

    def __init__(self, sino, angles, method, filter_name):
        if method not in ("fbp", "bpf", "dfi"):
            raise NotImplementedError(
                "method %r: this library reconstructs with 'fbp', 'bpf' or "
                "'dfi'" % (method,))
        self.nrow, self.ncol = sino.shape
        self.method, self.filter_name = method, filter_name
        self.sino = sino
        if method == "dfi":  # DFI takes the angles as given (None allowed)
            self.dfi_angles = angles
            return
        self.angles = R._validate(sino, 0.0, angles)[3]
        self.pad = min(int(0.15 * self.ncol), 150)
        if method == "fbp":
            f = R.filter_sinograms(sino.unsqueeze(1), self.pad, "edge", False,
                                   None, filter_name)
            self.src, self.src_rs = f, f.stride(0)
        else:
            src = sino if sino.stride(1) == 1 else sino.contiguous()
            self.src, self.src_rs = src, src.stride(0)
        self.trig = R._trig(self.angles, sino.device)

    def reconstruct(self, centers, ratio):
        """float32 [len(centers), ncol, ncol] reconstructions."""
        nrow, ncol, dev = self.nrow, self.ncol, self.sino.device
        if self.method == "dfi":
            from .dfi import dfi_reconstruction
            return torch.stack([dfi_reconstruction(
                self.sino, float(c), angles=self.dfi_angles, ratio=ratio,
                filter_name=self.filter_name, apply_log=False).to(
                    torch.float32) for c in centers])
        for c in centers:
            R._validate(self.sino, float(c), self.angles)
        out = torch.empty((len(centers), ncol, ncol), dtype=torch.float32,
                          device=dev)
        scale = R._scale(nrow)
        fbp = self.method == "fbp"
        keep = None
        masks = {R._mask_r2(ratio, float(c), ncol) if fbp else -1.0
                 for c in centers}
        groups = _centre_groups(centers) if len(masks) == 1 else None
        if groups is not None:
            # candidates a whole number of pixels apart: 4 per CTA
            mask_r2 = masks.pop()
            st = R._stream_ptr(dev)
            for r, ncls, c0, g, cnt in groups:
                nat.call("atb_backproject_centers", self.src.data_ptr(),
                         self.src_rs, nrow, ncol, self.trig.data_ptr(), c0,
                         g, cnt, 0 if fbp else 1, mask_r2,
                         scale if fbp else 1.0, out[r].data_ptr(),
                         out.stride(1), ncls * out.stride(0), 0, st)
        items = []
        for k, c in enumerate([] if groups is not None else centers):
            it = nat.BpItem()
            it.sino, it.sino_row_stride = self.src.data_ptr(), self.src_rs
            it.trig = self.trig.data_ptr()
            it.out, it.out_row_stride = out[k].data_ptr(), out.stride(1)
            it.center = float(np.float32(c))
            it.nrow, it.ncol = nrow, ncol
            if fbp:
                it.mask_r2, it.scale, it.edge_pad = R._mask_r2(
                    ratio, float(c), ncol), scale, 0
            else:
                it.mask_r2, it.scale, it.edge_pad = -1.0, 1.0, 1
            items.append(it)
        if items:
            keep = _backproject_items(items, dev, 1 if ncol <= 512 else 0)
        if not fbp:
            v = out.permute(1, 0, 2)  # [y, candidate, x], filtered in place
            R._circular_filter(v, None, self.filter_name, self.pad, "edge",
                               out=v)
            idx = torch.arange(ncol, device=dev) - ncol // 2
            d2 = (idx[None, :] ** 2 + idx[:, None] ** 2).to(torch.float64)
            for k, c in enumerate(centers):
                r2 = R._mask_r2(ratio, float(c), ncol)
                if r2 >= 0:
                    out[k] *= (d2 <= r2).to(out.dtype)
            out *= scale
        del keep
        return out


def reconstruct_centers(sino, centers, angles=None, method="fbp", ratio=1.0,
                        filter_name="hann"):
    """Reconstructions of one sinogram at several centres.

    ``sino``: 2-D float32 CUDA tensor, already in attenuation (-log) form.
    Returns a float32 [len(centers), ncol, ncol] CUDA tensor equal, slice by
    slice, to ``fbp_reconstruction`` / ``bpf_reconstruction`` (with
    ``apply_log=False`` and default pad) at each centre.
    """
    return _Source(sino, angles, method, filter_name).reconstruct(centers,
                                                                  ratio)


# --------------------------------------------------------------------------
# drop-in API
# --------------------------------------------------------------------------
def _prepare(sinogram, sigma, apply_log):
    """Smoothing and -log of ``reconstruction.py:1317-1325`` on the device.

    As in the reference, the replacement of values <= 0 by 1 happens in the
    array being searched: a fresh smoothed copy when ``sigma > 0``, the
    caller's own array otherwise.
    """
    if sigma > 0:
        t, _ = R._to_device(sinogram)
        if t.dim() != 2:
            raise ValueError("sinogram must be 2-D")
        t = gaussian_filter_rows(t, sigma, _integer_input(sinogram))
        if apply_log:
            R._check_log_input(t)
    else:
        if apply_log:
            R._check_log_input(sinogram)
        t, _ = R._to_device(sinogram)
        if t.dim() != 2:
            raise ValueError("sinogram must be 2-D")
    if apply_log:
        t = R._neg_log(t.unsqueeze(1))[:, 0, :]
    return t


def _find_center_based_slice_metric(sinogram, start, stop, step=1,
                                    metric="entropy", method="fbp", gpu=True,
                                    angles=None, ratio=1.0, filter_name="hann",
                                    apply_log=True, ncore=None,
                                    prefer="threads", sigma=2,
                                    return_metric=True, invert_metric=False,
                                    metric_function=None, **kwargs):
    """Metric of the reconstruction at every centre of
    ``np.arange(start, stop, step)``; ``reconstruction.py:1254-1346``.

    Returns ``(centers, metrics)`` if ``return_metric`` else the centre of
    the smallest metric.  ``gpu``, ``ncore`` and ``prefer`` are accepted
    for compatibility; the work always runs on the device.
    """
    list_center = np.arange(start, stop, step)
    num_center = len(list_center)
    if num_center == 0:
        raise ValueError("Invalid searching parameters: (start, stop, step)={}"
                         "!!!".format((start, stop, step)))
    sino = _prepare(sinogram, sigma, apply_log)
    ncol = sino.shape[1]
    source = _Source(sino, angles, method, filter_name)
    nmin, nmax = 0.0, 1.0
    if metric_function is None and metric == "entropy":
        img = source.reconstruct([np.mean(list_center)], ratio)[0]
        nmin, nmax = image_range(img)
        del img
        if nmin == nmax:
            raise ValueError("Empty image!!!")
    per_chunk = max(1, int(_CHUNK_BYTES // (4 * ncol * ncol)))
    list_metric = np.ones(num_center)
    for k0 in range(0, num_center, per_chunk):
        cs = list_center[k0:k0 + per_chunk]
        imgs = source.reconstruct(cs, ratio)
        if metric_function is None:
            m = "entropy" if metric == "entropy" else "sharpness"
            list_metric[k0:k0 + len(cs)] = slice_metrics(imgs, m, nmin, nmax)
        else:
            host = imgs.cpu().numpy()
            if method in ("bpf", "dfi"):
                host = host.astype(np.float64)
            for i in range(len(cs)):
                list_metric[k0 + i] = metric_function(host[i], **kwargs)
        del imgs
    if invert_metric:
        list_metric = np.max(list_metric) - list_metric
    opt_center = list_center[np.argmin(list_metric)]
    if return_metric:
        return list_center, list_metric
    return opt_center


def find_center_based_slice_metric(sinogram, start, stop, step=0.5,
                                   metric="entropy", radius=2, zoom=1.0,
                                   method="fbp", gpu=True, angles=None,
                                   ratio=1.0, filter_name="hann",
                                   apply_log=True, ncore=None, sigma=2,
                                   invert_metric=False, metric_function=None,
                                   **kwargs):
    """Centre of rotation from slice metrics; ``reconstruction.py:1349-1458``.

    A coarse pass at unit steps on the sinogram zoomed by ``zoom`` (device
    linear zoom), then a fine pass at ``step`` within ``radius`` of the
    coarse centre.  Metrics: ``"entropy"`` (histogram entropy) or
    ``"sharpness"``; a custom ``metric_function(recon, **kwargs)`` must be
    smallest at the best centre.
    """
    import scipy.ndimage as ndi
    zoom = np.clip(zoom, 0.01, 1.0)
    angles_zoom = angles
    t, _ = R._to_device(sinogram)
    sino_zoom = t.clone() if t is sinogram else t
    if zoom < 1.0:
        sino_zoom = zoom_image(t, zoom)
        start, stop = start * zoom, stop * zoom
        if angles is not None:
            # the angle table is host setup: scipy's own 1-D zoom
            a = angles.detach().cpu().numpy() if isinstance(
                angles, torch.Tensor) else np.asarray(angles)
            angles_zoom = ndi.zoom(np.tile(a, (1, 1)), (1.0, zoom))[0]
    del t
    kw = dict(metric=metric, method=method, gpu=gpu, ratio=ratio,
              filter_name=filter_name, apply_log=apply_log, ncore=ncore,
              sigma=sigma, return_metric=False, invert_metric=invert_metric,
              metric_function=metric_function)
    if stop > start:
        coarse_center = _find_center_based_slice_metric(
            sino_zoom, start, stop + 1, 1.0, angles=angles_zoom, **kw,
            **kwargs)
        coarse_center = coarse_center / zoom
    else:
        coarse_center = start / zoom
    del sino_zoom
    if radius != 0.0:
        radius = max(radius, step + 1.0 / zoom)
        start, stop = coarse_center - radius, coarse_center + radius + step
        center = _find_center_based_slice_metric(sinogram, start, stop, step,
                                                 angles=angles, **kw,
                                                 **kwargs)
    else:
        center = coarse_center
    return center


def _reconstruct_slice(sinogram, center, method, angles, ratio, filter_name,
                       apply_log, gpu, ncore):
    """One slice by ``method``; ``reconstruction.py:1177-1208``.  The
    ``astra`` and ``gridrec`` back-ends wrap external packages and raise
    ``NotImplementedError`` here."""
    if method == "fbp":
        return R.fbp_reconstruction(sinogram, center, angles=angles,
                                    ratio=ratio, filter_name=filter_name,
                                    apply_log=apply_log, gpu=gpu, ncore=ncore)
    if method == "bpf":
        return R.bpf_reconstruction(sinogram, center, angles=angles,
                                    ratio=ratio, filter_name=filter_name,
                                    apply_log=apply_log, gpu=gpu, ncore=ncore)
    if method in ("astra", "gridrec"):
        raise NotImplementedError(
            "method %r: this library reconstructs with 'fbp', 'bpf' or "
            "'dfi'" % (method,))
    from .dfi import dfi_reconstruction
    return dfi_reconstruction(sinogram, center, angles=angles, ratio=ratio,
                              filter_name=filter_name, apply_log=apply_log,
                              ncore=ncore)


def find_center_visual_slices(sinogram, output, start, stop, step=1,
                              zoom=0.5, method="fbp", gpu=False, angles=None,
                              ratio=1.0, filter_name="hann", apply_log=True,
                              ncore=None, display=False):
    """Reconstructions of a sinogram at candidate centres written as TIFF
    files ``center_<c>.tif`` into a new ``Find_center_<nnn>`` folder under
    ``output``, for choosing the centre by eye; ``reconstruction.py:
    1461-1533``.  The (zoomed) sinogram is filtered or ``-log``-ed once and
    every candidate is a work item of one persistent back-projection launch
    (``fbp`` / ``bpf``; ``dfi`` reconstructs candidate by candidate).
    Returns the folder path (with a trailing ``/``)."""
    import scipy.ndimage as ndi
    from ._files import make_folder_name, save_image
    output_name = make_folder_name(output, name_prefix="Find_center",
                                   zero_prefix=3)
    output_base = output + "/" + output_name + "/"
    (nrow, ncol) = sinogram.shape
    step = np.clip(step, 0.05, ncol - 1)
    start = np.clip(start, 0, ncol - 1)
    stop = np.clip(stop + step, start + step, ncol - 1)
    t, _ = R._to_device(sinogram)
    if t.dtype != torch.float32:
        t = t.to(torch.float32)
    if zoom != 1.0:
        t = zoom_image(t, zoom)
        start, stop, step = start * zoom, stop * zoom, step * zoom
        list_center = np.arange(start, stop, step)
        if angles is not None:
            # the angle table is host setup: scipy's own 1-D zoom
            a = angles.detach().cpu().numpy() if isinstance(
                angles, torch.Tensor) else np.asarray(angles)
            angles = ndi.zoom(np.tile(a, (1, 1)), (1.0, zoom))[0]
        sino = t
    else:
        list_center = np.arange(start, stop, step)
        sino = sinogram
    out_dtype = np.float32 if method == "fbp" else np.float64
    if method == "dfi":
        # DFI takes the logarithm after its sub-pixel centring shift, so
        # each candidate gets the transmission data (and its own warning)
        def chunks():
            for c in list_center:
                yield [c], _reconstruct_slice(
                    sino, c, method, angles, ratio, filter_name, apply_log,
                    gpu, ncore)[None]
    else:
        # -log once, with the reference's warning and in-place repair of
        # the array being reconstructed (the caller's own only without zoom)
        sino = _prepare(sino, 0, apply_log)
        source = _Source(sino, angles, method, filter_name)
        ncol1 = sino.shape[1]
        per_chunk = max(1, int(_CHUNK_BYTES // (4 * ncol1 * ncol1)))

        def chunks():
            for k0 in range(0, len(list_center), per_chunk):
                cs = list_center[k0:k0 + per_chunk]
                yield cs, source.reconstruct(cs, ratio)
    for cs, imgs in chunks():
        imgs = imgs.cpu().numpy() if isinstance(imgs, torch.Tensor) else \
            np.asarray(imgs)
        for center, img in zip(cs, imgs):
            file_name = "center_{0:.2f}".format(center / zoom) + ".tif"
            save_image(output_base + file_name, img.astype(out_dtype))
            if display:
                print("Done: {}".format(output_base + file_name))
    return output_base

