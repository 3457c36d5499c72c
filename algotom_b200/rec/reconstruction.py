"""Drop-in replacement of algotom's FBP / BPF reconstruction functions.

Same names, signatures, defaults, errors and warnings as
``algotom/rec/reconstruction.py`` (algotom 1.6.0) for the filtered
back-projection path; the compute runs in the sm_100a kernels of
``libalgotom_b200.so`` through its C ABI.  There is no CPU path: ``gpu`` and
``ncore`` are accepted for compatibility and do not change where the work
runs (``block`` is accepted and ignored; the kernels pick their own tiles).

Inputs may be NumPy arrays (results come back as NumPy arrays with the
reference's dtypes) or torch tensors (results stay torch tensors on the
tensor's CUDA device).  A few keyword-only extensions are available:
``out`` (write the reconstruction into a caller buffer, e.g. pinned host
memory), ``storage`` ("float32", "float16" or "bfloat16": the element type
of the filtered sinogram between the two kernels) and ``kahan`` ("chunk",
the default, or "angle").
"""
import math
import warnings

import numpy as np
import torch

from .. import _native as nat
from . import windows as win
from .windows import (make_smoothing_window, make_2d_ramp_window,  # noqa: F401
                      make_circular_ramp_window)

_STORAGE = {"float32": (torch.float32, nat.F32),
            "float16": (torch.float16, nat.F16),
            "bfloat16": (torch.bfloat16, nat.BF16)}

_spec_cache = {}
_tw_cache = {}


# --------------------------------------------------------------------------
# device plumbing
# --------------------------------------------------------------------------
def _device():
    if not torch.cuda.is_available():
        raise nat.NativeLibraryError(
            "algotom_b200 runs on a CUDA device only; none is available")
    return torch.device("cuda", torch.cuda.current_device())


def _stream_ptr(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def _to_device(x, device=None):
    """float32 CUDA tensor with a contiguous last axis; returns (t, is_np)."""
    if isinstance(x, torch.Tensor):
        dev = x.device if x.is_cuda else (device or _device())
        t = x.to(device=dev, dtype=torch.float32, non_blocking=True)
        is_np = False
    else:
        dev = device or _device()
        a = np.asarray(x)
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))
        t = t.to(dev, non_blocking=t.is_pinned())
        is_np = True
    if t.stride(-1) != 1:
        t = t.contiguous()
    return t, is_np


_trig_cache = {}


def _trig(angles, device):
    """(cos(-a), sin(-a)) in FP64 of the float32-rounded angles, as a
    device table kept for reuse: a repeated angle set costs neither the host
    trigonometry nor a host-to-device copy (which, from pageable memory,
    would also wait for the work already queued on the stream)."""
    a = np.float32(np.asarray(angles, dtype=np.float64))
    key = (a.tobytes(), str(device))
    t = _trig_cache.get(key)
    if t is not None:
        return t
    a = a.astype(np.float64)
    if not np.all(np.isfinite(a)):
        raise ValueError("angles must be finite")
    tab = np.stack([np.cos(-a), np.sin(-a)], axis=1)
    t = torch.from_numpy(np.ascontiguousarray(tab)).to(device)
    if len(_trig_cache) >= 16:
        _trig_cache.clear()
    _trig_cache[key] = t
    return t


def _twiddle(m, device):
    """Device twiddle table of the row filter's length-m transforms
    (``atb_filter_twiddles``: each FFT stage's twiddles in the order the
    kernel reads them, FP64-computed), cached per (m, device)."""
    key = (m, device)
    t = _tw_cache.get(key)
    if t is None:
        tw = np.empty(2 * m, dtype=np.float32)
        nat.call("atb_filter_twiddles", int(m), tw.ctypes.data)
        t = torch.from_numpy(tw).to(device)
        _tw_cache[key] = t
    return t


def _spectrum(ramp_win, filter_name, nrow, ncol, pad, m, device):
    """Device spectrum [1 or nrow, m] for the row filter (transform length
    m from ``atb_filter_length``)."""
    n = ncol + 2 * pad
    if ramp_win is None or np.shape(ramp_win) != (nrow, n):
        key = (filter_name, ncol, pad, m, device)
        t = _spec_cache.get(key)
        if t is None:
            sp = win.row_filter_spectrum(win.ramp_window_row(n, filter_name),
                                         ncol, pad, m)
            t = torch.from_numpy(sp.view(np.float32).copy()).to(device)
            if len(_spec_cache) > 32:
                _spec_cache.clear()
            _spec_cache[key] = t
        return t, 1
    rw = np.asarray(ramp_win.cpu() if isinstance(ramp_win, torch.Tensor)
                    else ramp_win)
    rows = rw[:1] if np.all(rw == rw[:1]) else rw
    sp = win.row_filter_spectrum(rows, ncol, pad, m)
    return torch.from_numpy(sp.view(np.float32).copy()).to(device), len(rows)


def _as3(t):
    """[nrow, ncol] -> [nrow, 1, ncol] view."""
    return t.unsqueeze(1) if t.dim() == 2 else t


def filter_sinograms(sino3, pad, pad_mode="edge", apply_log=False,
                     ramp_win=None, filter_name="hann", storage="float32"):
    """Device ramp filter of a [nrow, nslice, ncol] float32 CUDA tensor.

    Returns a new [nrow, nslice, ncol] tensor of ``storage`` type.
    """
    nrow, nslice, ncol = sino3.shape
    if pad_mode not in nat.PAD_MODES:
        raise ValueError("pad_mode %r is not supported" % (pad_mode,))
    m = nat.call("atb_filter_length", int(ncol), int(pad))
    dev = sino3.device
    spec, spec_rows = _spectrum(ramp_win, filter_name, nrow, ncol, pad, m,
                                dev)
    tdtype, code = _STORAGE[storage]
    out = torch.empty((nrow, nslice, ncol), dtype=tdtype, device=dev)
    nat.call("atb_filter_rows", sino3.data_ptr(), sino3.stride(0),
             sino3.stride(1), nrow, nslice, ncol, int(pad),
             nat.PAD_MODES[pad_mode], int(bool(apply_log)), spec.data_ptr(),
             spec_rows, _twiddle(m, dev).data_ptr(), m,
             out.data_ptr(), code, out.stride(0), out.stride(1),
             _stream_ptr(dev))
    return out


def backproject(sino3, angles, center, edge_pad=False, mask_r2=-1.0,
                scale=1.0, out=None, kahan="chunk", trig=None, variant=0,
                staging="tma"):
    """Device back-projection of [nrow, nslice, ncol] -> [ncol, nslice, ncol].

    ``sino3`` may be float32, float16 or bfloat16 (last axis contiguous).
    ``trig`` may hold the angle table from :func:`_trig` already on the
    device (saves its host-to-device copy per call).  ``variant`` selects
    the single-slice tile variant (0: 64 x 64, 1: 32 x 32).  ``staging``:
    "tma" stages the detector windows of 2- and 4-slice CTAs with TMA box
    loads where the rows are 16-byte aligned, "cp.async" always with
    cp.async; the results are the same.
    """
    if staging not in ("tma", "cp.async"):
        raise ValueError("staging must be 'tma' or 'cp.async'")
    nrow, nslice, ncol = sino3.shape
    dev = sino3.device
    code = {torch.float32: nat.F32, torch.float16: nat.F16,
            torch.bfloat16: nat.BF16}[sino3.dtype]
    if trig is None:
        trig = _trig(angles, dev)
    if out is None:
        out = torch.empty((ncol, nslice, ncol), dtype=torch.float32,
                          device=dev)
    nat.call("atb_backproject", sino3.data_ptr(), code, sino3.stride(0),
             sino3.stride(1), nrow, nslice, ncol, trig.data_ptr(),
             float(np.float32(center)), int(bool(edge_pad)), float(mask_r2),
             float(scale), out.data_ptr(), out.stride(0), out.stride(1),
             (1 if kahan == "angle" else 0) | (int(variant) << 2) |
             (16 if staging == "cp.async" else 0), _stream_ptr(dev))
    return out


def _backproject_tuned(f, angles, center, **kw):
    """Back-projection of a single slice with the autotuned tile variant."""
    from .autotune import tuned_single_variant
    nrow, nslice, ncol = f.shape
    if nslice != 1 or kw.get("kahan") == "angle":
        return backproject(f, angles, center, **kw)
    trig = _trig(angles, f.device)
    out = torch.empty((ncol, 1, ncol), dtype=torch.float32, device=f.device)
    v = tuned_single_variant(ncol, nrow, lambda var: backproject(
        f, angles, center, out=out, trig=trig, variant=var, **kw))
    return backproject(f, angles, center, out=out, trig=trig, variant=v, **kw)


def _neg_log(sino3):
    out = torch.empty_like(sino3)
    nrow, nslice, ncol = sino3.shape
    nat.call("atb_neg_log", sino3.data_ptr(), sino3.stride(0),
             sino3.stride(1), nrow, nslice, ncol, out.data_ptr(),
             out.stride(0), out.stride(1), _stream_ptr(sino3.device))
    return out


def _check_log_input(sinogram):
    """Reference pre-step (``reconstruction.py:431-436``): warn on values
    <= 0 and set them to 1 in the caller's array."""
    if isinstance(sinogram, torch.Tensor):
        bad = sinogram <= 0.0
        if bool(bad.any()):
            warnings.warn("!!!Applying logarithm is enabled but "
                          "there are values <= 0.0 in the data!!!")
            sinogram.masked_fill_(bad, 1.0)
    else:
        if np.any(sinogram <= 0.0):
            warnings.warn("!!!Applying logarithm is enabled but "
                          "there are values <= 0.0 in the data!!!")
            sinogram[sinogram <= 0.0] = np.float32(1.0)


def _validate(sinogram, center, angles):
    shape = tuple(sinogram.shape)
    if len(shape) == 3:
        nrow, nslice, ncol = shape
    elif len(shape) == 2:
        (nrow, ncol), nslice = shape, 1
    else:
        raise ValueError("sinogram must be 2-D or 3-D")
    if center < 0 or center >= ncol:
        raise ValueError("Center is out of the range [0, {}]".format(ncol - 1))
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, nrow))
    else:
        if len(angles) != nrow:
            raise ValueError("!!!Number of angles is not the same as the row "
                             "number of the sinogram!!!")
        if isinstance(angles, torch.Tensor):
            angles = angles.detach().cpu().numpy()
    return nrow, nslice, ncol, np.asarray(angles, dtype=np.float64)


def _mask_r2(ratio, center, ncol):
    if ratio is None:
        return -1.0
    if ratio == 0.0:
        ratio = min(center, ncol - center) / (0.5 * ncol)
    radius = ratio * (ncol // 2)
    return float(radius * radius)


def _scale(nrow):
    with np.errstate(divide="ignore", invalid="ignore"):
        return float(np.float32(np.pi) / np.float32(nrow - 1))


def _finish(rec3, two_d, is_np, out, np_dtype=np.float32):
    """Shape and hand back a [ncol, nslice, ncol] device result."""
    res = rec3[:, 0, :] if two_d else rec3
    if out is not None:
        dst = out if isinstance(out, torch.Tensor) else torch.from_numpy(out)
        if tuple(dst.shape) != tuple(res.shape):
            raise ValueError("out has shape %s, expected %s"
                             % (tuple(dst.shape), tuple(res.shape)))
        # pinned host memory (e.g. torch pin_memory) gets a direct DMA
        dst.copy_(res, non_blocking=dst.is_cuda or dst.is_pinned())
        if not dst.is_cuda:
            torch.cuda.current_stream(res.device).synchronize()
        return out
    if is_np:
        return res.cpu().numpy().astype(np_dtype, copy=False)
    return res


# --------------------------------------------------------------------------
# public drop-in API (algotom.rec.reconstruction names)
# --------------------------------------------------------------------------
def apply_ramp_filter(sinogram, ramp_win=None, filter_name=None, pad=None,
                      pad_mode="edge"):
    """Ramp filter of a 2-D sinogram; ``reconstruction.py:118-153``.

    NumPy input returns float64 like the reference; tensors stay float32
    on the device.
    """
    t, is_np = _to_device(sinogram)
    nrow, ncol = t.shape
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    f = filter_sinograms(_as3(t), pad, pad_mode, False, ramp_win, filter_name)
    f = f[:, 0, :]
    return f.cpu().numpy().astype(np.float64) if is_np else f


def back_projection_gpu(sinogram, angles, center, block=(16, 16),
                        edge_pad=False):
    """Back-projection of one sinogram; ``reconstruction.py:193-226``."""
    t, is_np = _to_device(sinogram)
    rec = backproject(_as3(t), angles, center, edge_pad=edge_pad)
    return _finish(rec, True, is_np, None)


def back_projection_gpu_chunk(sinograms, angles, center, block=(16, 16),
                              edge_pad=False):
    """Back-projection of [nrow, nslice, ncol]; ``reconstruction.py:267-304``."""
    t, is_np = _to_device(sinograms)
    rec = backproject(t, angles, center, edge_pad=edge_pad)
    return _finish(rec, False, is_np, None)


def back_projection_cpu(sinogram, angles, center, edge_pad=False):
    """Name kept from ``reconstruction.py:307-359``; runs on the device."""
    return back_projection_gpu(sinogram, angles, center, edge_pad=edge_pad)


SLAB = 32  # slices per slab when a host stack is streamed through the device


def _host_tensor(x):
    """C-contiguous float32 CPU tensor sharing the caller's memory when it
    can (NumPy array or CPU tensor)."""
    if isinstance(x, torch.Tensor):
        t = x.detach()
        if t.dtype != torch.float32 or not t.is_contiguous():
            t = t.to(torch.float32).contiguous()
        return t
    a = np.asarray(x)
    if a.dtype != np.float32 or not a.flags.c_contiguous:
        a = np.ascontiguousarray(a, dtype=np.float32)
    return torch.from_numpy(a)


def _slab_spans(nslice, slab):
    """(first slice, count) of the slabs of a streamed stack: full slabs of
    ``slab``, with the first and last ramped (slab/4, slab/4, slab/2) so the
    copy-in that nothing overlaps before the first kernel and the copy-out
    after the last one are short."""
    ramp = [max(1, slab // 4), max(1, slab // 4), max(1, slab // 2)]
    if nslice < 2 * slab + 2 * sum(ramp):
        sizes = [slab] * (nslice // slab) + ([nslice % slab]
                                            if nslice % slab else [])
    else:
        mid = nslice - 2 * sum(ramp)
        sizes = ramp + [slab] * (mid // slab) + \
            ([mid % slab] if mid % slab else []) + ramp[::-1]
    spans, k0 = [], 0
    for n in sizes:
        spans.append((k0, n))
        k0 += n
    return spans


def _resume_key(shape, center, angles, mask_r2, scale, ramp_win,
                filter_name, pad, pad_mode, apply_log, storage, kahan, slab):
    """What defines a streamed reconstruction's result, for its manifest."""
    import hashlib
    ang = np.ascontiguousarray(np.float32(angles)).tobytes()
    win = None
    if ramp_win is not None:
        w = ramp_win.cpu().numpy() if isinstance(ramp_win, torch.Tensor) \
            else np.asarray(ramp_win)
        win = hashlib.sha1(np.ascontiguousarray(w).tobytes()).hexdigest()
    return {"shape": [int(v) for v in shape],
            "center": float(np.float32(center)),
            "angles_sha1": hashlib.sha1(ang).hexdigest(),
            "mask_r2": float(mask_r2), "scale": float(scale),
            "ramp_win_sha1": win, "filter_name": filter_name,
            "pad": int(pad), "pad_mode": pad_mode,
            "apply_log": bool(apply_log), "storage": storage,
            "kahan": kahan, "slab": int(slab)}


def _fbp_streamed(host, center, angles, mask_r2, scale, ramp_win, filter_name,
                  pad, pad_mode, apply_log, out_host, storage, kahan,
                  slab=SLAB, manifest=None):
    """FBP of a host stack [nrow, nslice, ncol] streamed through the device
    in slabs of up to ``slab`` slices (ramped at both ends): while slab k is
    filtered and back-projected, slab k+1 is copied in and slab k-1 copied
    out (one copy stream each way, double-buffered, ordered by events).
    With a :class:`~algotom_b200.rec.resume.SlabManifest`, slabs it lists
    are skipped and every slab whose copy-out has completed is recorded."""
    nrow, nslice, ncol = host.shape
    dev = _device()
    k_sl = max(1, min(slab, nslice))
    spans = _slab_spans(nslice, k_sl)
    if manifest is not None:
        spans = [sp for sp in spans if not manifest.is_done(sp)]
    pending = []  # (copy-out event, span) not yet recorded as finished
    cmp = torch.cuda.current_stream(dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    in_buf = [torch.empty((nrow, k_sl, ncol), dtype=torch.float32, device=dev)
              for _ in range(2)]
    out_buf = [torch.empty((ncol, k_sl, ncol), dtype=torch.float32,
                           device=dev) for _ in range(2)]
    for t in in_buf:
        t.record_stream(s_in)
    for t in out_buf:
        t.record_stream(s_out)
    ev_in_ready = [torch.cuda.Event() for _ in range(2)]
    ev_in_free = [torch.cuda.Event() for _ in range(2)]
    ev_out_ready = [torch.cuda.Event() for _ in range(2)]
    ev_out_free = [torch.cuda.Event() for _ in range(2)]
    row_b, slab_b = nslice * ncol * 4, k_sl * ncol * 4
    hp, op = host.data_ptr(), out_host.data_ptr()
    trig = _trig(angles, dev)
    cmp.synchronize()
    for k, (k0, kk) in enumerate(spans):
        b = k % 2
        if manifest is not None and pending:
            fin = [sp for ev, sp in pending if ev.query()]
            pending = [(ev, sp) for ev, sp in pending if not ev.query()]
            manifest.mark(fin)
        if k >= 2:
            s_in.wait_event(ev_in_free[b])
        nat.call("atb_copy_2d", in_buf[b].data_ptr(), slab_b, hp + k0 * ncol * 4,
                 row_b, kk * ncol * 4, nrow, 0, s_in.cuda_stream)
        ev_in_ready[b].record(s_in)
        cmp.wait_event(ev_in_ready[b])
        f = filter_sinograms(in_buf[b][:, :kk, :], pad, pad_mode, apply_log,
                             ramp_win, filter_name, storage)
        ev_in_free[b].record(cmp)
        if k >= 2:
            cmp.wait_event(ev_out_free[b])
        backproject(f, angles, center, edge_pad=False, mask_r2=mask_r2,
                    scale=scale, out=out_buf[b][:, :kk, :], kahan=kahan,
                    trig=trig)
        ev_out_ready[b].record(cmp)
        s_out.wait_event(ev_out_ready[b])
        nat.call("atb_copy_2d", op + k0 * ncol * 4, row_b, out_buf[b].data_ptr(),
                 slab_b, kk * ncol * 4, ncol, 1, s_out.cuda_stream)
        ev_out_free[b].record(s_out)
        if manifest is not None:
            done = torch.cuda.Event()
            done.record(s_out)
            pending.append((done, (k0, kk)))
        del f
    s_out.synchronize()
    s_in.synchronize()
    if manifest is not None:
        manifest.mark([sp for _, sp in pending])
    return out_host


def fbp_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       ramp_win=None, filter_name="hann", pad=None,
                       pad_mode="edge", apply_log=True, gpu=True,
                       block=(16, 16), ncore=None, *, out=None,
                       storage="float32", kahan="chunk", resume=None):
    """FBP of a 2-D [nrow, ncol] or 3-D [nrow, nslice, ncol] sinogram.

    Drop-in for ``algotom.rec.reconstruction.fbp_reconstruction``
    (``reconstruction.py:362-493``): -log (with the in-place <= 0 -> 1
    replacement and warning), padded ramp-and-window filter, back-projection
    without edge padding, circle mask (``ratio``; 0.0 picks the largest disc
    inside the centred field), scale pi/(nrow-1).  Returns float32
    [ncol, ncol] or [ncol, nslice, ncol].

    ``resume`` (a file path; host stacks with a persistent ``out``, e.g. a
    ``numpy.memmap``): record every finished slab in that JSON manifest and
    skip the slabs it already lists, so a run cut short is completed by
    calling again with the same arguments (``rec/resume.py``).
    """
    nrow, nslice, ncol, angles = _validate(sinogram, center, angles)
    if apply_log:
        _check_log_input(sinogram)
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    on_host = not (isinstance(sinogram, torch.Tensor) and sinogram.is_cuda)
    if resume is not None and not (on_host and len(sinogram.shape) == 3
                                   and out is not None):
        raise ValueError("resume needs a host 3-D stack and a persistent "
                         "out array that holds the finished slices")
    if on_host and len(sinogram.shape) == 3:
        # host stack: stream slabs through the device, overlapping copies
        host = _host_tensor(sinogram)
        if out is None:
            res = torch.empty((ncol, nslice, ncol), dtype=torch.float32,
                              pin_memory=True)
        else:
            res = out if isinstance(out, torch.Tensor) else \
                torch.from_numpy(out)
            if tuple(res.shape) != (ncol, nslice, ncol) or \
                    res.dtype != torch.float32 or not res.is_contiguous():
                raise ValueError("out must be a C-contiguous float32 array "
                                 "of shape %s" % ((ncol, nslice, ncol),))
        manifest = None
        if resume is not None:
            from .resume import SlabManifest
            manifest = SlabManifest.open(str(resume), _resume_key(
                host.shape, center, angles, _mask_r2(ratio, center, ncol),
                _scale(nrow), ramp_win, filter_name, pad, pad_mode,
                apply_log, storage, kahan, SLAB))
        _fbp_streamed(host, center, angles, _mask_r2(ratio, center, ncol),
                      _scale(nrow), ramp_win, filter_name, pad, pad_mode,
                      apply_log, res, storage, kahan, manifest=manifest)
        if out is not None:
            return out
        return res if isinstance(sinogram, torch.Tensor) else res.numpy()
    t, is_np = _to_device(sinogram)
    two_d = t.dim() == 2
    f = filter_sinograms(_as3(t), pad, pad_mode, apply_log, ramp_win,
                         filter_name, storage)
    del t
    rec = _backproject_tuned(f, angles, center, edge_pad=False,
                             mask_r2=_mask_r2(ratio, center, ncol),
                             scale=_scale(nrow), kahan=kahan)
    del f
    return _finish(rec, two_d, is_np, out)


def apply_circular_ramp_filter(rec_img, ramp_win=None, filter_name=None,
                               pad=None, pad_mode="edge"):
    """2-D circular ramp filter; ``reconstruction.py:527-560``.

    ``real(ifft2(fft2(pad(x)) * ifftshift(W2)))`` cropped.  NumPy input
    returns float64 like the reference.
    """
    t, is_np = _to_device(rec_img)
    ncol = t.shape[0]
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    r = _circular_filter(t.to(torch.float32)[:, None, :], ramp_win,
                         filter_name, pad, pad_mode)[:, 0, :]
    return r.cpu().numpy().astype(np.float64) if is_np else r


_circ_cache = {}


def _circular_spectrum(ramp_win, filter_name, ncol, pad, device):
    """Spectrum, its kind and the twiddles of ``atb_bpf_filter2d`` for the
    2-D circular ramp filter of ``reconstruction.py:527-560``.

    The reference keeps ``real(ifft2(fft2(x) * H))`` with
    ``H = ifftshift(W2)``; for a real image only the Hermitian part
    ``Hh = (H[k] + conj(H[-k])) / 2`` reaches the real part.  For the
    library's transform length T = N = ncol + 2 pad the spectrum is Hh
    itself (real when W2 is); for a longer T (N with a prime factor above
    13) it is the transform of the N-periodic kernel ``ifft2(Hh)`` laid on
    the T-torus at the lags ``[pad - N + 1, pad + ncol - 1]`` that the crop
    uses.  Either way scaled by 1 / T^2 and stored transposed ([kx][ky]).
    Returns (spectrum, is_complex, twiddle, T), cached per (filter, ncol,
    pad, device) for the built-in windows.
    """
    n = ncol + 2 * pad
    key = None
    if ramp_win is None or np.shape(ramp_win) != (n, n):
        key = (filter_name, ncol, pad, str(device))
        hit = _circ_cache.get(key)
        if hit is not None:
            return hit
        ramp_win = make_circular_ramp_window(n, filter_name)
    t = nat.call("atb_bpf_filter2d_length", ncol, pad)
    w2 = ramp_win.cpu().numpy() if isinstance(ramp_win, torch.Tensor) \
        else np.asarray(ramp_win)
    h = np.fft.ifftshift(np.asarray(w2, dtype=np.complex128))
    hm = np.roll(np.flip(h, axis=(0, 1)), 1, axis=(0, 1))  # H[-k1, -k2]
    hh = 0.5 * (h + np.conj(hm))
    if t == n:
        spec = hh / float(n) ** 2
        if not np.any(spec.imag):
            spec = spec.real
    else:
        k = np.fft.ifft2(hh).real  # real: hh is Hermitian
        lag = np.arange(pad - n + 1, pad + ncol)
        km = np.zeros((t, t))
        km[np.ix_(lag % t, lag % t)] = k[np.ix_(lag % n, lag % n)]
        spec = np.fft.fft2(km) / float(t) ** 2
    is_complex = np.iscomplexobj(spec)
    sp = torch.from_numpy(np.ascontiguousarray(spec.T)).to(
        device, torch.complex128 if is_complex else torch.float64)
    tw = torch.from_numpy(np.exp(-2j * np.pi * np.arange(t) / t)).to(
        device, torch.complex128)
    res = (sp, is_complex, tw, t)
    if key is not None:
        if len(_circ_cache) > 8:
            _circ_cache.clear()
        _circ_cache[key] = res
    return res


# device bytes of 2-D transform workspace per call of the BPF filter
_BPF_WORKSPACE = 2 << 30


def _circular_filter(stack, ramp_win, filter_name, pad, pad_mode, out=None,
                     mask_r2=-1.0, scale=1.0):
    """2-D circular ramp filter of ``reconstruction.py:527-560`` on every
    slice of a back-projection stack ``[ncol (y), nslice, ncol (x)]``
    (any strides, x contiguous), with the circle mask and scale of
    ``reconstruction.py:679-684`` fused: ``atb_bpf_filter2d`` (numpy's ten
    pad modes, FP64 transforms of this library).  ``out`` may be ``stack``
    itself."""
    ncol, nslice, _ = stack.shape
    if pad_mode not in nat.PAD_MODES:
        raise ValueError("pad_mode %r is not supported" % (pad_mode,))
    if stack.stride(-1) != 1:
        stack = stack.contiguous()
    spec, is_complex, tw, t = _circular_spectrum(ramp_win, filter_name, ncol,
                                                 pad, stack.device)
    if out is None:
        out = torch.empty_like(stack)
    one = nat.call("atb_bpf_filter2d_workspace", ncol, pad, 1)
    npairs = (nslice + 1) // 2
    pairs = max(1, min(npairs, _BPF_WORKSPACE // one))
    nbytes = nat.call("atb_bpf_filter2d_workspace", ncol, pad, pairs)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=stack.device)
    nat.call("atb_bpf_filter2d", stack.data_ptr(), stack.stride(0),
             stack.stride(1), nslice, ncol, pad, nat.PAD_MODES[pad_mode],
             spec.data_ptr(), int(is_complex), tw.data_ptr(), float(mask_r2),
             float(scale), out.data_ptr(), out.stride(0), out.stride(1),
             ws.data_ptr(), nbytes, _stream_ptr(stack.device))
    return out


def bpf_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       ramp_win=None, filter_name="hann", pad=None,
                       pad_mode="edge", apply_log=True, gpu=True,
                       block=(16, 16), ncore=None, *, out=None,
                       kahan="chunk"):
    """BPF of a 2-D or 3-D sinogram; ``reconstruction.py:563-684``.

    -log, back-projection of the unfiltered sinogram with edge padding, 2-D
    circular ramp filter per slice, mask, scale pi/(nrow-1).  2-D NumPy
    input returns float64 (as the reference does), 3-D float32.
    """
    nrow, nslice, ncol, angles = _validate(sinogram, center, angles)
    if apply_log:
        _check_log_input(sinogram)
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    t, is_np = _to_device(sinogram)
    two_d = t.dim() == 2
    s3 = _neg_log(_as3(t)) if apply_log else _as3(t)
    bp = backproject(s3, angles, center, edge_pad=True, kahan=kahan)
    del s3, t
    # filter, mask and scale in place, in the [ncol][nslice][ncol] layout
    rec = _circular_filter(bp, ramp_win, filter_name, pad, pad_mode, out=bp,
                           mask_r2=_mask_r2(ratio, center, ncol),
                           scale=_scale(nrow))
    return _finish(rec, two_d, is_np, out,
                   np.float64 if two_d else np.float32)


# centre search by slice metrics (reconstruction.py:1254-1458), kept in this
# module's namespace like the reference's
from .center import (find_center_based_slice_metric,  # noqa: E402,F401
                     _find_center_based_slice_metric, _reconstruct_slice,
                     find_center_visual_slices)

# direct Fourier inversion (reconstruction.py:687-907)
from .dfi import (dfi_reconstruction,  # noqa: E402,F401
                  generate_mapping_coordinate)
