"""Drop-in replacement of algotom's vertical-slice reconstruction.

Same names, signatures, defaults, errors and warnings as
``algotom/rec/vertrec.py`` (algotom 1.6.0) for the vertical back-projectors
(``:53-335``), the slice-line geometry (``:338-447``) and the three
vertical reconstructions (``:450-1252``); the compute runs in the sm_100a
kernels of ``libalgotom_b200.so``:

- ``atb_flat_log``: flat/dark correction and ``-log`` of each chunk of
  projections (the reference's warning texts, and its in-place repair of
  values <= 0 in the caller's array when no flat field is given);
- ``atb_filter_rows``: the ramp filter of every projection row
  (``ramp_filter="before"``);
- ``atb_vertical_backproject``: the gather, all slices of a call at once,
  accumulated in FP64 across chunks.

The ramp filter applied after the back-projection (``"after"``) runs in
FP64 on the device (``atb_filter_rows64``, see :func:`_after_filter64`).

Projections may be NumPy arrays, array-likes with NumPy slicing (e.g. HDF5
datasets) or torch tensors; the reference's chunks of ``chunk_size``
projections are grouped into device slabs of about 512 MB that are cropped
and copied to the device in turn (CUDA tensors are used in place).  As in
algotom, ``gpu=True`` back-projects positions from float32-rounded angles,
points and centre (what the reference's GPU kernels receive) and
``gpu=False`` from their FP64 values (the reference's CPU kernels); both run
on the device.  ``block``, ``ncore`` and ``prefer`` are accepted and ignored.
"""
import sys
import time
import warnings

import numpy as np
import torch

from .. import _native as nat
from . import reconstruction as R
from . import windows as win
from .center import _gaussian_weights, _integer_input, slice_metrics

_WARN_FULL = ("!!! Applying logarithm is enabled but there are values <= 0.0"
              " in the data !!!")
_WARN_REST = "Applying logarithm is enabled but there are values <= 0.0."


# --------------------------------------------------------------------------
# slice-line geometry (vertrec.py:338-447; defines the points, kept alike)
# --------------------------------------------------------------------------
def _get_points_single_line(slice_index, alpha, width):
    """x and y coordinates of the points of a vertical slice at angle alpha
    (degrees) through image column ``slice_index``; ``vertrec.py:338-384``.
    """
    if alpha < 0.0 or alpha > 180.0:
        raise ValueError("Angle is out of range [0, 180] (degree)")
    if slice_index < 0 or slice_index > width - 1:
        raise ValueError(f"Slice index is out of range [0, {width - 1}]")
    center = np.ceil(0.5 * (width - 1))
    x_min, x_max = - center, width - center
    y_min, y_max = x_min, x_max
    angle = np.deg2rad(alpha)
    x0 = y0 = slice_index - center
    if alpha <= 45 or alpha >= 135:
        a_fact = np.tan(angle)
        # the reference tests the angle in radians against 45 here, which
        # always holds, so both halves of this branch use -y0 / cos
        b_fact = - y0 / np.cos(angle)
        xcr = - a_fact * b_fact / (1 + a_fact ** 2)
        xlist = xcr + np.arange(x_min, x_max) * np.cos(angle)
        ylist = a_fact * xlist + b_fact
    else:
        a_fact = np.cos(angle) / np.sin(angle)
        # likewise (radians against 90): always x0 / sin
        b_fact = x0 / np.sin(angle)
        ycr = - a_fact * b_fact / (1 + a_fact ** 2)
        ylist = ycr + np.arange(y_min, y_max) * np.sin(angle)
        xlist = a_fact * ylist + b_fact
    return xlist, ylist


def _get_points_multiple_lines(start_index, stop_index, alpha, width,
                               step_index=1):
    """Points of parallel slices ``start_index..stop_index`` (float32
    [nslice, npts] each); ``vertrec.py:387-418``."""
    x_mat, y_mat = [], []
    for idx in np.arange(start_index, stop_index + 1, step_index):
        xlist, ylist = _get_points_single_line(idx, alpha, width)
        x_mat.append(xlist)
        y_mat.append(ylist)
    return np.float32(x_mat), np.float32(y_mat)


def _get_points_multiple_lines_different_angles(list_index, list_alpha,
                                                width):
    """Points of slices at their own angles; ``vertrec.py:421-447``."""
    x_mat, y_mat = [], []
    for i, index in enumerate(list_index):
        xlist, ylist = _get_points_single_line(index, list_alpha[i], width)
        x_mat.append(xlist)
        y_mat.append(ylist)
    return np.float32(x_mat), np.float32(y_mat)


# --------------------------------------------------------------------------
# device steps
# --------------------------------------------------------------------------
def _trig_plus(angles, device, round32):
    """(cos a, sin a) in FP64, of float32-rounded angles when ``round32``."""
    a = np.asarray(angles.detach().cpu() if isinstance(angles, torch.Tensor)
                   else angles, dtype=np.float64)
    if round32:
        a = np.float32(a).astype(np.float64)
    tab = np.stack([np.cos(a), np.sin(a)], axis=1)
    return torch.from_numpy(np.ascontiguousarray(tab)).to(device)


def _points(x_mat, y_mat, width, device, round32):
    """float64 [nline, width, 2] device table of (x, y)."""
    x = np.atleast_2d(np.asarray(x_mat, dtype=np.float64))
    y = np.atleast_2d(np.asarray(y_mat, dtype=np.float64))
    if x.shape != y.shape:
        raise ValueError("x and y coordinates differ in shape")
    if x.shape[1] < width:
        raise ValueError("%d points per slice for an image width of %d"
                         % (x.shape[1], width))
    x, y = x[:, :width], y[:, :width]
    if round32:
        x = np.float32(x).astype(np.float64)
        y = np.float32(y).astype(np.float64)
    return torch.from_numpy(np.ascontiguousarray(np.stack([x, y], -1))).to(
        device)


def _backproject(proj, trig, pts, center, edge_pad, acc):
    """acc [nline, height, npts] += vertical back-projection of the float32
    CUDA slab ``proj`` [n, height, width] (last axis contiguous), with
    scratch for the split of the angles over CTAs when the output is small.
    ``center``: a number, or a float64 CUDA tensor with one centre per
    line."""
    n, height, width = proj.shape
    nline, npts = pts.shape[0], pts.shape[1]
    nbytes = nat.call("atb_vertical_workspace", n, height, npts, nline)
    work = torch.empty(int(nbytes), dtype=torch.uint8, device=proj.device) \
        if nbytes > 0 else None
    per_line = isinstance(center, torch.Tensor)
    nat.call("atb_vertical_backproject", proj.data_ptr(), proj.stride(0),
             proj.stride(1), n, height, width, trig.data_ptr(),
             pts.data_ptr(), npts, npts, nline,
             0.0 if per_line else float(center),
             center.data_ptr() if per_line else None,
             int(bool(edge_pad)), acc.data_ptr(), acc.stride(0),
             acc.stride(1), work.data_ptr() if work is not None else None,
             int(nbytes), R._stream_ptr(proj.device))


def _flat_log(raw, code, dark, flat_dark, apply_log, out, nonpos):
    n, height, width = raw.shape
    nat.call("atb_flat_log", raw.data_ptr(), code, raw.stride(0),
             raw.stride(1), n, height, width,
             dark.data_ptr() if dark is not None else None,
             flat_dark.data_ptr() if flat_dark is not None else None,
             dark.stride(0) if dark is not None else 0, int(bool(apply_log)),
             out.data_ptr(), out.stride(0), out.stride(1), nonpos.data_ptr(),
             R._stream_ptr(raw.device))


def _filter_rows(x3, pad, pad_mode, spec, flen, out3):
    """Row filter of a float32 [nrow, nslice, ncol] CUDA view into out3."""
    nrow, nslice, ncol = x3.shape
    dev = x3.device
    nat.call("atb_filter_rows", x3.data_ptr(), x3.stride(0), x3.stride(1),
             nrow, nslice, ncol, int(pad), nat.PAD_MODES[pad_mode], 0,
             spec.data_ptr(), 1, R._twiddle(flen, dev).data_ptr(), flen,
             out3.data_ptr(), nat.F32, out3.stride(0), out3.stride(1),
             R._stream_ptr(dev))


_AFTER_CACHE = {}
_TW_CACHE = {}


def _twiddle64(t, device):
    """complex128 exp(-2 pi i m / t), m < t, on ``device`` (cached)."""
    key = (t, str(device))
    tw = _TW_CACHE.get(key)
    if tw is None:
        if len(_TW_CACHE) > 8:
            _TW_CACHE.clear()
        tw = _TW_CACHE[key] = torch.from_numpy(
            np.exp(-2j * np.pi * np.arange(t) / t)).to(device,
                                                         torch.complex128)
    return tw


def _after_spectrum(filter_name, width, pad, device):
    """(spectrum, twiddle, T) of ``atb_filter_rows64`` for the after filter:
    the kernel real(ifft(ifftshift(|W|))) of the padded width N, laid on
    the length-T circle at the lags [pad - N + 1, pad + width - 1] the crop
    uses (the kernel itself when T = N), transformed and scaled by 1 / T;
    FP64, cached per (filter, width, pad, device)."""
    key = (filter_name, width, pad, str(device))
    hit = _AFTER_CACHE.get(key)
    if hit is not None:
        return hit
    n = width + 2 * pad
    t = nat.call("atb_filter_rows64_length", int(width), int(pad))
    h = np.fft.ifftshift(np.abs(win.ramp_window_row(n, filter_name)))
    kappa = np.real(np.fft.ifft(h))
    if t == n:
        b = kappa
    else:
        lags = np.arange(pad - n + 1, pad + width)
        b = np.zeros(t)
        b[lags % t] = kappa[lags % n]
    spec = torch.from_numpy(np.fft.fft(b) / t).to(device, torch.complex128)
    tw = _twiddle64(t, device)
    if len(_AFTER_CACHE) > 8:
        _AFTER_CACHE.clear()
    hit = _AFTER_CACHE[key] = (spec, tw, t)
    return hit


def _after_filter64(ver, filter_name, pad, pad_mode):
    """The ramp filter applied to every row of the vertical slices after
    the back-projection (``vertrec.py:684-688``, ``:698-706``):
    ``real(ifft(ifftshift(fftshift(fft(pad(row))) * |W|)))`` cropped, in
    FP64 (``atb_filter_rows64``: padding in NumPy's modes, one row per
    transform, so equal rows give equal results as NumPy's do) from the
    FP64 back-projection sums.  The ramp filter
    removes the large smooth part of those sums, so a float32 transform (or
    float32 input) would lose ~1e-4 of the result.  ``ver``: float64
    [nline, height, width]; returns float64."""
    nline, height, width = ver.shape
    if pad_mode not in nat.PAD_MODES:
        raise ValueError("pad_mode %r is not supported" % (pad_mode,))
    spec, tw, t = _after_spectrum(filter_name, width, pad, ver.device)
    rows = ver.reshape(-1, width)
    if rows.stride(-1) != 1:
        rows = rows.contiguous()
    stat = None
    if pad > 0 and nat.PAD_MODES[pad_mode] >= nat.PAD_MODES["mean"]:
        if pad_mode == "mean":
            stat = rows.mean(dim=1)
        elif pad_mode == "maximum":
            stat = rows.amax(dim=1)
        elif pad_mode == "minimum":
            stat = rows.amin(dim=1)
        else:
            srt = torch.sort(rows, dim=1).values
            stat = 0.5 * (srt[:, (width - 1) // 2] + srt[:, width // 2])
        stat = stat.contiguous()
    out = torch.empty_like(rows)
    nat.call("atb_filter_rows64", rows.data_ptr(), rows.stride(0),
             rows.shape[0], width, int(pad), nat.PAD_MODES[pad_mode],
             stat.data_ptr() if stat is not None else None, spec.data_ptr(),
             tw.data_ptr(), t, out.data_ptr(), out.stride(0),
             R._stream_ptr(ver.device))
    return out.reshape(nline, height, width)


# --------------------------------------------------------------------------
# vertical back-projectors (vertrec.py:53-335)
# --------------------------------------------------------------------------
def vertical_back_projection_cpu(projections, angles, xlist, ylist, center,
                                 edge_pad=False):
    """Vertical back-projection of a [depth, height, width] projection
    stack onto the points (xlist, ylist); ``vertrec.py:53-109``.  FP64
    positions; runs on the device.  Returns float32 (height, width)."""
    return _vbp_api(projections, angles, xlist, ylist, center, edge_pad,
                    round32=False, single=True)


def vertical_back_projection_gpu(projections, angles, xlist, ylist, center,
                                 edge_pad=False, block=(16, 16)):
    """As :func:`vertical_back_projection_cpu` with float32-rounded angles,
    points and centre; ``vertrec.py:215-252``."""
    return _vbp_api(projections, angles, xlist, ylist, center, edge_pad,
                    round32=True, single=True)


def vertical_back_projection_cpu_chunk(projections, angles, x_mat, y_mat,
                                       center, edge_pad=False):
    """Several slices, one per row of (x_mat, y_mat); ``vertrec.py:112-172``.
    Returns float32 (num_slice, height, width)."""
    return _vbp_api(projections, angles, x_mat, y_mat, center, edge_pad,
                    round32=False, single=False)


def vertical_back_projection_gpu_chunk(projections, angles, x_mat, y_mat,
                                       center, edge_pad=False,
                                       block=(16, 16)):
    """As :func:`vertical_back_projection_cpu_chunk` with float32-rounded
    inputs; ``vertrec.py:295-335``."""
    return _vbp_api(projections, angles, x_mat, y_mat, center, edge_pad,
                    round32=True, single=False)


def _vbp_api(projections, angles, xs, ys, center, edge_pad, round32,
             single):
    t, is_np = R._to_device(projections)
    if t.dim() != 3:
        raise ValueError("projections must be 3-D (depth, height, width)")
    depth, height, width = t.shape
    if len(angles) != depth:
        raise ValueError("%d angles for %d projections" % (len(angles),
                                                           depth))
    dev = t.device
    trig = _trig_plus(angles, dev, round32)
    pts = _points(xs, ys, width, dev, round32)
    c = float(np.float32(center)) if round32 else float(center)
    acc = torch.zeros((pts.shape[0], height, width), dtype=torch.float64,
                      device=dev)
    _backproject(t, trig, pts, c, edge_pad, acc)
    res = acc.to(torch.float32)
    if single:
        res = res[0]
    return res.cpu().numpy() if is_np else res


# --------------------------------------------------------------------------
# chunked vertical reconstruction (vertrec.py:450-1252)
# --------------------------------------------------------------------------
class _Chunks:
    """Cropped slabs of projections as float32-or-uint16 CUDA tensors.

    CUDA sources are used in place (views).  Host sources go to the device
    through a copy stream and two device buffers, so the copy of slab k+1
    overlaps the kernels of slab k: pinned host memory (torch pinned tensors
    or NumPy views of them) by strided DMA, one 2-D copy per slab or per
    projection; other arrays (and HDF5 datasets) through two pinned staging
    buffers."""

    def __init__(self, projections, top, bot, left, right, device):
        self.src = projections
        self.box = (top, bot, left, right)
        self.dev = device
        self.cuda = isinstance(projections, torch.Tensor) and \
            projections.is_cuda
        self.stream = None if self.cuda else torch.cuda.Stream(device)
        self.pinned = None
        if not self.cuda:
            t = self._as_torch(projections)
            if t is not None and t.dim() == 3 and t.stride(2) == 1 and \
                    t.dtype in (torch.float32, torch.uint16) and \
                    t.is_pinned():
                self.pinned = t
        self.buffers = {}
        self.copied = [None, None]  # slot's host-to-device copy finished
        self.freed = [None, None]   # slot's kernels finished

    @staticmethod
    def _as_torch(x):
        if isinstance(x, torch.Tensor):
            return x
        if isinstance(x, np.ndarray) and x.dtype in (np.float32, np.uint16) \
                and all(st >= 0 for st in x.strides):
            return torch.from_numpy(x)
        return None

    def _host_view(self, start, stop):
        top, bot, left, right = self.box
        v = self.src[start:stop, top:bot, left:right]
        if isinstance(v, torch.Tensor):
            v = v.numpy()
        v = np.asarray(v)
        if v.dtype not in (np.float32, np.uint16):
            v = v.astype(np.float32)
        return v

    def _slot_buffers(self, slot, shape, tdt, staging):
        key = (slot, tdt, shape, staging)
        buf = self.buffers.get(key)
        if buf is None:
            self.buffers = {kk: bb for kk, bb in self.buffers.items()
                            if kk[0] != slot}
            host = torch.empty(shape, dtype=tdt, pin_memory=True) \
                if staging else None
            buf = (host, torch.empty(shape, dtype=tdt, device=self.dev))
            self.buffers[key] = buf
        return buf

    def fetch(self, k, start, stop):
        """Slab [start, stop) on the device (slot k % 2) and its dtype code."""
        top, bot, left, right = self.box
        if self.cuda:
            v = self.src[start:stop, top:bot, left:right]
            if v.dtype not in (torch.float32, torch.uint16):
                v = v.to(torch.float32)
            if v.stride(-1) != 1:
                v = v.contiguous()
            return v, nat.U16 if v.dtype == torch.uint16 else nat.F32
        slot = k % 2
        cur = torch.cuda.current_stream(self.dev)
        shape = (stop - start, bot - top, right - left)
        if self.pinned is not None:
            t = self.pinned
            _, dev = self._slot_buffers(slot, shape, t.dtype, False)
        else:
            v = self._host_view(start, stop)
            tdt = torch.uint16 if v.dtype == np.uint16 else torch.float32
            host, dev = self._slot_buffers(slot, shape, tdt, True)
            if self.copied[slot] is not None:
                self.copied[slot].synchronize()  # staging buffer free again
            np.copyto(host.numpy(), v)
        if self.freed[slot] is not None:
            self.stream.wait_event(self.freed[slot])
        if self.pinned is not None:
            es = t.element_size()
            sp, sr = t.stride(0), t.stride(1)
            h, w = shape[1], shape[2]
            st = self.stream.cuda_stream
            base = t.data_ptr() + (start * sp + top * sr + left) * es
            if sp == t.shape[1] * sr and h == t.shape[1]:
                # whole projections: the slab's rows are evenly spaced
                nat.call("atb_copy_2d", dev.data_ptr(), w * es, base, sr * es,
                         w * es, shape[0] * h, 0, st)
            else:
                for q in range(shape[0]):
                    nat.call("atb_copy_2d", dev[q].data_ptr(), w * es,
                             base + q * sp * es, sr * es, w * es, h, 0, st)
        else:
            with torch.cuda.stream(self.stream):
                dev.copy_(host, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.copied[slot] = ev
        cur.wait_event(ev)
        return dev, nat.U16 if dev.dtype == torch.uint16 else nat.F32

    def done(self, k):
        """Slab k's kernels are queued: its slot is free after them."""
        if not self.cuda:
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream(self.dev))
            self.freed[k % 2] = ev

    def repair(self, start, stop):
        """The reference's in-place <= 0 -> 1 on the caller's chunk view
        (no flat field: its chunk is a view of the caller's array)."""
        top, bot, left, right = self.box
        v = self.src[start:stop, top:bot, left:right]
        if isinstance(v, torch.Tensor):
            v.masked_fill_(v <= 0, 1)
        elif isinstance(v, np.ndarray) and v.flags.writeable:
            v[v <= 0.0] = np.float32(1.0)


def _slabs(spans, chunk_bytes, cuda_src, preprocess, target=1 << 29):
    """Group consecutive reference chunks into device slabs: all of them for
    a CUDA source that needs no pre-step, else about ``target`` bytes."""
    if cuda_src and not preprocess:
        return [(0, len(spans))]
    per = max(1, int(target // max(1, chunk_bytes)))
    return [(k, min(k + per, len(spans))) for k in range(0, len(spans), per)]


def _check_common(projections, center, angles, crop, proj_start, proj_stop,
                  ramp_filter):
    """The shared argument checks of the three reconstructions."""
    if not (ramp_filter == "before" or ramp_filter == "after"
            or ramp_filter is None):
        raise ValueError("Must use one of these options: "
                         "'before', 'after', None")
    (num_proj0, height0, width0) = projections.shape
    if proj_stop == -1:
        proj_stop = num_proj0
    num_proj = proj_stop - proj_start
    if num_proj < 1:
        raise ValueError("Wrong value of proj_start or proj_stop !!! Given "
                         "the number of projections {}".format(num_proj0))
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, num_proj))
    else:
        if len(angles) != num_proj:
            raise ValueError("!!! Number of angles is not the same as the "
                             "number of projections !!!")
    (cr_top, cr_bottom, cr_left, cr_right) = crop
    top, bot = cr_top, height0 - cr_bottom
    left, right = cr_left, width0 - cr_right
    width = right - left
    height = bot - top
    if height < 1 or width < 1:
        raise ValueError("Can't crop images with the given parameters !!!")
    if center < 0 or center > (width - 1):
        raise ValueError("Center (relative to the cropped image) is out of "
                         "range {})".format((0, width - 1)))
    return (num_proj0, height0, width0, proj_stop, num_proj, angles, top,
            bot, left, right, width, height)


def _fields(flat_field, dark_field, height0, width0, top, bot, left, right):
    """(dark, flat - dark with zeros set to 1) cropped, float32 NumPy, or
    (None, None); ``vertrec.py:561-583``."""
    if (flat_field is None) and (dark_field is None):
        return None, None
    if flat_field is None:
        flat_field = np.ones((height0, width0), dtype=np.float32)
    else:
        if flat_field.shape != (height0, width0):
            raise ValueError("!!! Shape of flat-field and projection-image"
                             " is not the same !!!")
    if dark_field is None:
        dark_field = np.zeros((height0, width0), dtype=np.float32)
    else:
        if dark_field.shape != (height0, width0):
            raise ValueError("!!! Shape of dark-field and projection-image"
                             " is not the same !!!")
    flat = np.asarray(flat_field)[top:bot, left:right]
    dark = np.asarray(dark_field)[top:bot, left:right]
    flat_dark = flat - dark
    flat_dark[flat_dark == 0.0] = np.float32(1.0)
    return np.float32(dark), np.float32(flat_dark)


def _gaussian_slab(x, wts, tmp, out, to_int=False):
    """``gaussian_filter(x, (0, sigma, sigma))`` of a float32 CUDA slab
    [n, height, width] (last axis contiguous) into ``out``: down the
    columns into ``tmp``, then along the rows; float32 between the passes,
    as scipy.  ``to_int``: integer counts, each pass truncated toward zero
    (scipy's result for an integer array)."""
    n, height, width = x.shape
    r = wts.numel() - 1
    st = R._stream_ptr(x.device)
    ti = int(bool(to_int))
    nat.call("atb_gaussian_cols", x.data_ptr(), x.stride(0), x.stride(1), n,
             height, width, wts.data_ptr(), r, tmp.data_ptr(), tmp.stride(0),
             tmp.stride(1), ti, st)
    nat.call("atb_gaussian_rows", tmp.data_ptr(), width, n * height, width,
             wts.data_ptr(), r, out.data_ptr(), width, ti, st)


def _reconstruct(projections, x_mat, y_mat, center, geo, flat_field,
                 dark_field, chunk_size, ramp_filter, filter_name, pad,
                 pad_mode, apply_log, gpu, show_progress, masking,
                 round_points, line_centers=None, sigma=0.0,
                 log_warning=None, device_out=False):
    """The chunk loop of ``vertrec.py:584-695`` for any set of slices;
    returns float64 [num_slice, height, width] (NumPy for host input unless
    ``device_out``).

    ``line_centers``: one centre per slice instead of ``center``.
    ``sigma`` > 0: each projection is smoothed first (the Gaussian of a
    centre search, ``vertrec.py:1348-1349``).  ``log_warning``: one warning
    with this text if ``-log`` met values <= 0 anywhere, instead of the
    reconstructions' per-chunk warnings ("": no warning)."""
    (num_proj0, height0, width0, proj_stop, num_proj, angles, top, bot,
     left, right, width, height) = geo
    proj_start = proj_stop - num_proj
    dark_np, flat_dark_np = _fields(flat_field, dark_field, height0, width0,
                                    top, bot, left, right)
    if chunk_size is None:
        chunk_size = min(30, num_proj // 4 + 1)
    if chunk_size > num_proj or chunk_size < 1:
        chunk_size = num_proj
    num_iter = num_proj // chunk_size
    num_rest = num_proj - num_iter * chunk_size
    if pad is None:
        pad = min(int(0.15 * width), 150)
    edge_pad = ramp_filter != "before"
    is_cuda = isinstance(projections, torch.Tensor) and projections.is_cuda
    dev = projections.device if is_cuda else R._device()
    if pad_mode not in nat.PAD_MODES:
        raise ValueError("pad_mode %r is not supported" % (pad_mode,))

    dark = flat_dark = None
    if dark_np is not None:
        dark = torch.from_numpy(dark_np).to(dev)
        flat_dark = torch.from_numpy(flat_dark_np).to(dev)
    trig = _trig_plus(angles, dev, gpu)
    pts = _points(x_mat, y_mat, width, dev, gpu or round_points)
    c = float(np.float32(center)) if gpu else float(center)
    if line_centers is not None:
        lc = np.asarray(line_centers, dtype=np.float64)
        if gpu:
            lc = np.float32(lc).astype(np.float64)
        c = torch.from_numpy(np.ascontiguousarray(lc)).to(dev)
    nline = pts.shape[0]
    wts = None
    if sigma > 0:
        wts = torch.from_numpy(_gaussian_weights(sigma)).to(dev)
        to_int = _integer_input(projections)
    acc = torch.zeros((nline, height, width), dtype=torch.float64,
                      device=dev)
    flen = nat.call("atb_filter_length", int(width), int(pad))
    spec_before = None
    if ramp_filter == "before":
        spec_before, _ = R._spectrum(None, filter_name, height, width, pad,
                                     flen, dev)
    spans = [(i * chunk_size + proj_start, (i + 1) * chunk_size + proj_start)
             for i in range(num_iter)]
    if num_rest != 0:
        start = num_iter * chunk_size + proj_start
        spans.append((start, start + num_rest))
    nonpos = torch.zeros(len(spans), dtype=torch.int32, device=dev)
    chunks = _Chunks(projections, top, bot, left, right, dev)
    preprocess = apply_log or dark is not None or wts is not None
    item = 4 if chunks.pinned is None else chunks.pinned.element_size()
    slabs = _slabs(spans, chunk_size * height * width * item, is_cuda,
                   preprocess or (is_cuda and projections.dtype !=
                                  torch.float32))
    work = {}
    if show_progress:
        t0 = time.time()
    for q, (k0, k1) in enumerate(slabs):
        s0, s1 = spans[k0][0], spans[k1 - 1][1]
        raw, code = chunks.fetch(q, s0, s1)
        n = s1 - s0
        if code == nat.F32 and not preprocess:
            pre = raw  # nothing to correct: back-project the slab as it is
        else:
            pre = work.get(("pre", n))
            if pre is None:
                pre = torch.empty((n, height, width), dtype=torch.float32,
                                  device=dev)
                work[("pre", n)] = pre
            if wts is not None:
                tmp = work.get(("tmp", n))
                if tmp is None:
                    tmp = torch.empty_like(pre)
                    work[("tmp", n)] = tmp
                if code != nat.F32:  # counts to float32 first
                    _flat_log(raw, code, None, None, False, pre, nonpos[:1])
                    raw = pre
                _gaussian_slab(raw, wts, tmp, pre, to_int)
                raw, code = pre, nat.F32
            for k in range(k0, k1):  # one warning counter per chunk
                if raw is pre and not apply_log and dark is None:
                    break  # smoothed, nothing else to do
                a, b = spans[k][0] - s0, spans[k][1] - s0
                _flat_log(raw[a:b], code, dark, flat_dark, apply_log,
                          pre[a:b], nonpos[k:k + 1])
        src = pre
        if ramp_filter == "before":
            filt = work.get(("filt", n))
            if filt is None:
                filt = torch.empty_like(pre)
                work[("filt", n)] = filt
            _filter_rows(pre, pad, pad_mode, spec_before, flen, filt)
            src = filt
        _backproject(src, trig[s0 - proj_start:s1 - proj_start], pts, c,
                     edge_pad, acc)
        chunks.done(q)
        if show_progress:
            torch.cuda.current_stream(dev).synchronize()
            elapsed_time = time.time() - t0
            percent_complete = 100.0 * (s1 - proj_start) / num_proj
            sys.stdout.write(f"\rProcessed {s1 - proj_start}/{num_proj} "
                             f"images ({percent_complete:.0f}%) - "
                             f"Time elapsed: {elapsed_time:.2f} seconds")
            sys.stdout.flush()
    if ramp_filter == "after":
        ver = _after_filter64(acc, filter_name, pad, pad_mode)
    else:
        ver = acc
    del acc
    if apply_log:
        counts = nonpos.cpu().numpy()
        if log_warning and counts.any():
            warnings.warn(log_warning)
        for k, (start, stop) in enumerate(spans):
            if counts[k] > 0:
                if log_warning is None:
                    warnings.warn(_WARN_FULL if k < num_iter else _WARN_REST)
                if dark is None and wts is None:
                    chunks.repair(start, stop)
    if show_progress:
        print("\nDone! Total time elapsed: {0:.2f}".format(time.time() - t0))
    if masking:
        rad = int(min(center, width - center))
        pad_left = (width - 2 * rad) // 2
        m = torch.zeros(width, dtype=ver.dtype, device=dev)
        m[pad_left:pad_left + 2 * rad] = 1.0
        ver = ver * m
    ver = (ver * np.pi) / (num_proj - 1)
    return ver if is_cuda or device_out else ver.cpu().numpy()


def _as_dtype(x, np_dtype):
    if isinstance(x, torch.Tensor):
        return x.to(torch.float64 if np_dtype == np.float64
                    else torch.float32)
    return x.astype(np_dtype, copy=False)


def vertical_reconstruction(projections, slice_index, center, alpha=0.0,
                            flat_field=None, dark_field=None, angles=None,
                            crop=(0, 0, 0, 0), proj_start=0, proj_stop=-1,
                            chunk_size=30, ramp_filter="after",
                            filter_name="hann", pad=None, pad_mode="edge",
                            apply_log=True, gpu=True, block=(16, 16),
                            ncore=None, prefer="threads", show_progress=True,
                            masking=False):
    """Reconstruct one vertical slice from projections (depth, height,
    width); ``vertrec.py:450-695``.  Returns (height, width): float64 after
    the "after" ramp filter (as the reference), float32 otherwise."""
    geo = _check_common(projections, center, angles, crop, proj_start,
                        proj_stop, ramp_filter)
    width = geo[10]
    if slice_index < 0 or slice_index > (width - 1):
        raise ValueError("Index (relative to the cropped image) is out of "
                         "range {})".format((0, width - 1)))
    xlist, ylist = _get_points_single_line(slice_index, alpha, width)
    ver = _reconstruct(projections, xlist, ylist, center, geo, flat_field,
                       dark_field, chunk_size, ramp_filter, filter_name, pad,
                       pad_mode, apply_log, gpu, show_progress, masking,
                       round_points=False)[0]
    return _as_dtype(ver, np.float64 if ramp_filter == "after"
                     else np.float32)


def vertical_reconstruction_multiple(projections, start_index, stop_index,
                                     center, alpha=0.0, step_index=1,
                                     flat_field=None, dark_field=None,
                                     angles=None, crop=(0, 0, 0, 0),
                                     proj_start=0, proj_stop=-1, chunk_size=30,
                                     ramp_filter="after", filter_name="hann",
                                     pad=None, pad_mode="edge", apply_log=True,
                                     gpu=True, block=(16, 16), ncore=None,
                                     prefer="threads", show_progress=True,
                                     masking=False):
    """Reconstruct parallel vertical slices ``start_index..stop_index`` at
    angle ``alpha``; ``vertrec.py:709-977``.  Returns float32
    (num_slice, height, width)."""
    geo = _check_common(projections, center, angles, crop, proj_start,
                        proj_stop, ramp_filter)
    width = geo[10]
    if start_index < 0 or start_index > (width - 1):
        raise ValueError("Start index (relative to the cropped image) is out "
                         "of range {})".format((0, width - 1)))
    if stop_index == -1:
        stop_index = width - 1
    if stop_index < 0 or stop_index > (width - 1):
        raise ValueError("Start index (relative to the cropped image) is out "
                         "of range {})".format((0, width - 1)))
    x_mat, y_mat = _get_points_multiple_lines(start_index, stop_index, alpha,
                                              width, step_index)
    return _as_dtype(_reconstruct(
        projections, x_mat, y_mat, center, geo, flat_field, dark_field,
        chunk_size, ramp_filter, filter_name, pad, pad_mode, apply_log, gpu,
        show_progress, masking, round_points=True), np.float32)


def vertical_reconstruction_different_angles(projections, slice_indices,
                                             alphas, center, flat_field=None,
                                             dark_field=None, angles=None,
                                             crop=(0, 0, 0, 0), proj_start=0,
                                             proj_stop=-1, chunk_size=30,
                                             ramp_filter="after",
                                             filter_name="hann", pad=None,
                                             pad_mode="edge", apply_log=True,
                                             gpu=True, block=(16, 16),
                                             ncore=None, prefer="threads",
                                             show_progress=True,
                                             masking=False):
    """Reconstruct vertical slices each at its own index and angle;
    ``vertrec.py:980-1252``.  Returns float32 (num_slice, height, width)."""
    if len(slice_indices) != len(alphas):
        raise ValueError("!!! Number of slice indices is not the same as the "
                         "number of angles !!!")
    geo = _check_common(projections, center, angles, crop, proj_start,
                        proj_stop, ramp_filter)
    width1 = geo[10] - 1
    if any(idx < 0 or idx > width1 for idx in slice_indices):
        raise ValueError("Slice index (relative to the cropped image) is out "
                         "of range {})".format((0, width1)))
    x_mat, y_mat = _get_points_multiple_lines_different_angles(
        slice_indices, alphas, geo[10])
    return _as_dtype(_reconstruct(
        projections, x_mat, y_mat, center, geo, flat_field, dark_field,
        chunk_size, ramp_filter, filter_name, pad, pad_mode, apply_log, gpu,
        show_progress, masking, round_points=True), np.float32)


# --------------------------------------------------------------------------
# centre search on a vertical slice (vertrec.py:1255-1383)
# --------------------------------------------------------------------------
_SEARCH_BYTES = 4 << 30  # FP64 slices reconstructed per pass over the data


def _autocorrelation(imgs):
    """``mean(max(|ifft(|fft(row)|^2)|, axis=1))`` of every float32 image
    of [n, rows, cols] (``vertrec.py:1255-1261``): the row maxima by
    ``atb_autocorr_rowmax`` (FP64 transforms), their mean per image in
    NumPy as the reference takes it.  Widths with no transform length up to
    7168 (a prime factor above 13 and more than 3584 columns) take the
    library FFT."""
    n, rows, cols = imgs.shape
    t = nat.load().atb_autocorr_length(int(cols))
    if t < 0:
        f = torch.fft.fft(imgs, dim=-1)
        ac = torch.fft.ifft(f.abs() ** 2, dim=-1).abs()
        return ac.amax(dim=-1).to(torch.float64).mean(dim=-1).cpu().numpy()
    x = imgs.reshape(n * rows, cols)
    if x.stride(-1) != 1:
        x = x.contiguous()
    tw = _twiddle64(t, imgs.device)
    out = torch.empty(n * rows, dtype=torch.float64, device=imgs.device)
    nat.call("atb_autocorr_rowmax", x.data_ptr(), x.stride(0), n * rows,
             cols, tw.data_ptr(), t, out.data_ptr(),
             R._stream_ptr(imgs.device))
    return out.cpu().numpy().reshape(n, rows).mean(axis=1)


def _entropy(imgs, nmin, nmax):
    """Histogram entropy of [n, rows, cols] slices normalised by
    (nmin, nmax), in the slices' precision."""
    if imgs.dtype == torch.float32:
        return slice_metrics(imgs, "entropy", nmin, nmax)
    imgs = imgs.contiguous()
    n, rows, cols = imgs.shape
    nbytes = nat.call("atb_slice_metric_workspace", n, rows, cols,
                      nat.METRICS["entropy"])
    work = torch.empty(int(nbytes), dtype=torch.uint8, device=imgs.device)
    out = torch.empty(n, dtype=torch.float64, device=imgs.device)
    nat.call("atb_slice_entropy64", imgs.data_ptr(), imgs.stride(0),
             imgs.stride(1), n, rows, cols, float(nmin), float(nmax),
             work.data_ptr(), work.numel(), out.data_ptr(),
             R._stream_ptr(imgs.device))
    return out.cpu().numpy()


def _candidate_slices(projections, slice_index, centers, alpha, angles,
                      chunk_size, ramp_filter, sigma, apply_log, gpu):
    """Yield ``(first, slices)`` for consecutive groups of ``centers``: the
    vertical slice at ``slice_index`` / ``alpha`` reconstructed at each
    centre as the searches' ``vertical_reconstruction`` calls make it (hann
    window, pad min(0.15 width, 150), edge mode, no mask, ``-log`` in the
    smoothing pass), every centre of a group a line of the same launch;
    float64 CUDA tensors after the "after" ramp filter, float32 otherwise.
    The reconstructions' own argument checks run first, for every centre."""
    (num_proj, height, width) = projections.shape
    geo = None
    for cen in centers:
        geo = _check_common(projections, cen, angles, (0, 0, 0, 0), 0, -1,
                            ramp_filter)
    if slice_index < 0 or slice_index > (width - 1):
        raise ValueError("Index (relative to the cropped image) is out of "
                         "range {})".format((0, width - 1)))
    pad = min(int(0.15 * width), 150)
    xlist, ylist = _get_points_single_line(slice_index, alpha, width)
    out_dtype = torch.float64 if ramp_filter == "after" else torch.float32
    log_text = ("!!! Applying logarithm is enabled but there are values "
                "<= 0.0 in the data !!!")
    per_pass = max(1, int(_SEARCH_BYTES // (8 * height * width)))
    for g0 in range(0, len(centers), per_pass):
        group = centers[g0:g0 + per_pass]
        xs = np.tile(np.asarray(xlist), (len(group), 1))
        ys = np.tile(np.asarray(ylist), (len(group), 1))
        recs = _reconstruct(
            projections, xs, ys, group[0], geo, None, None, chunk_size,
            ramp_filter, "hann", pad, "edge", apply_log, gpu, False, False,
            round_points=False, line_centers=group, sigma=sigma,
            log_warning=log_text if g0 == 0 else "", device_out=True)
        yield g0, recs.to(out_dtype)


def _search_mask(list_center, width):
    """The mask of the smallest candidate centre (vertrec.py:1355-1361)."""
    rad = int(min(np.min(list_center), width - np.min(list_center)))
    pad_left = (width - 2 * rad) // 2
    pad_right = width - 2 * rad - pad_left
    return np.pad(np.ones(2 * rad, dtype=np.float32), (pad_left, pad_right),
                  mode="constant")


def find_center_vertical_slice(projections, slice_index, start, stop,
                               step=1.0, metric="entropy", alpha=0.0,
                               angles=None, chunk_size=30,
                               ramp_filter="after", sigma=3, apply_log=True,
                               gpu=True, block=(16, 16), ncore=None,
                               prefer="threads", show_progress=True,
                               masking=True, return_metric=False,
                               invert_metric=False, metric_function=None,
                               **kwargs):
    """Centre of rotation from metrics of one vertical slice reconstructed
    at every centre of ``np.arange(start, stop + step, step)``;
    ``vertrec.py:1264-1383``.

    The projections are smoothed (``sigma``; integer projections such as
    uint16 counts truncated toward zero after each pass, as scipy stores
    them) and ``-log``-ed on the device chunk by chunk.  Integer counts with
    ``apply_log=False`` and the "after" filter are back-projected as float32;
    the reference's CPU back-projector would interpolate them in the integer
    type and wrap around.  Every candidate centre -- plus the mean centre that
    sets the entropy's normalisation -- is a line of the same vertical
    back-projection launch, so the data are read once for all of them
    (in passes of about 4 GB of FP64 slices when there are many).  Metrics:
    ``"entropy"``, ``"sharpness"``, ``"autocorrelation"`` (device
    kernels) or ``metric_function(recon, **kwargs)`` on each slice as a
    NumPy array.  Returns the centre of the smallest metric, or
    ``(list_center, list_metric)`` with ``return_metric``.
    """
    if (metric != "entropy" and metric != "sharpness"
            and metric != "autocorrelation" and metric_function is None):
        msg = "Please select one of three options: 'entropy', 'sharpness', " \
              "'autocorrelation'; or provide a custom method."
        raise ValueError(msg)
    if ramp_filter is None:
        ramp_filter = "after"
    list_center = np.arange(start, stop + step, step)
    list_metric = np.zeros_like(list_center)
    num_metric = len(list_metric)
    (num_proj, height, width) = projections.shape
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, num_proj))
    use_entropy = metric_function is None and metric == "entropy"
    centers = ([np.mean(list_center)] if use_entropy else []) + \
        list(list_center)
    mask = _search_mask(list_center, width) if masking else None
    nmin = nmax = None
    if show_progress:
        t0 = time.time()
    done = 0
    for g0, recs in _candidate_slices(projections, slice_index, centers,
                                      alpha, angles, chunk_size, ramp_filter,
                                      sigma, apply_log, gpu):
        if use_entropy and g0 == 0:
            first = recs[0]
            if recs.dtype == torch.float32:
                nmin = np.float32(first.min().item())
                nmax = np.float32(first.max().item())
            else:
                nmin, nmax = first.min().item(), first.max().item()
            recs = recs[1:]
        if mask is not None:
            recs = recs * torch.from_numpy(mask).to(recs.device).to(
                recs.dtype)
        k = len(recs)
        if k == 0:
            continue
        if metric_function is not None:
            host = recs.cpu().numpy()
            values = [metric_function(host[i], **kwargs) for i in range(k)]
        elif metric == "entropy":
            values = _entropy(recs, nmin, nmax)
        elif metric == "autocorrelation":
            values = _autocorrelation(recs.to(torch.float32))
        else:
            values = slice_metrics(recs.to(torch.float32), "sharpness")
        for i in range(k):
            list_metric[done + i] = values[i]
            if show_progress:
                elapsed_time = time.time() - t0
                percent_complete = 100.0 * (done + i + 1) / num_metric
                sys.stdout.write(
                    f"\rReconstructed image using the center: "
                    f"{list_center[done + i]}. "
                    f"Progress: {percent_complete:.0f}% - "
                    f"Time elapsed: {elapsed_time:.2f} seconds")
        done += k
        del recs
    if invert_metric:
        list_metric = np.max(list_metric) - list_metric
    min_pos = np.argmin(list_metric)
    center = list_center[min_pos]
    if show_progress:
        print("\nDone! Optimal center: {0}.".format(center))
    if return_metric is True:
        return list_center, list_metric
    else:
        return center


def find_center_visual_vertical_slices(projections, output_folder,
                                       slice_index, start, stop, step=1.0,
                                       alpha=0.0, angles=None, chunk_size=30,
                                       ramp_filter="after", apply_log=True,
                                       gpu=True, block=(16, 16), ncore=None,
                                       prefer="processes", display=True,
                                       masking=True):
    """The vertical slice reconstructed at every centre of
    ``np.arange(start, stop + step, step)`` written as TIFF files
    ``center_<c>.tif`` into a new ``Find_center_<nnn>`` folder under
    ``output_folder``, for choosing the centre by eye;
    ``vertrec.py:1431-1535``.  ``-log`` runs chunk by chunk on the device
    (with the reference's warning and in-place repair), and every candidate
    is a line of the same vertical back-projection launch.  Returns the
    folder path (with a trailing ``/``)."""
    from ._files import make_folder_name, save_image
    output_name = make_folder_name(output_folder, name_prefix="Find_center",
                                   zero_prefix=3)
    output_base = output_folder + "/" + output_name + "/"
    list_center = np.arange(start, stop + step, step)
    (num_proj, height, width) = projections.shape
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, num_proj))
    if ramp_filter is None:
        ramp_filter = "after"
    mask = _search_mask(list_center, width) if masking else None
    if display:
        t0 = time.time()
    for g0, recs in _candidate_slices(projections, slice_index,
                                      list(list_center), alpha, angles,
                                      chunk_size, ramp_filter, 0, apply_log,
                                      gpu):
        host = recs.cpu().numpy()
        for i, recon in enumerate(host):
            if mask is not None:
                recon = recon * mask
            center = list_center[g0 + i]
            file_name = "center_{0:.2f}".format(center) + ".tif"
            save_image(output_base + file_name, recon)
            if display:
                print("Done: {0}. Time elapsed {1:.2f}".format(
                    output_base + file_name, time.time() - t0))
    return output_base

