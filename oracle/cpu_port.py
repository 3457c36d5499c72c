"""CPU port of the reference path -- TEST INFRASTRUCTURE ONLY.

ctypes binding of ``liboracle_bp.so`` (``bp_port.c``) plus a CPU FBP driver
that mirrors ``fbp_reconstruction(..., gpu=False)``
(``algotom/rec/reconstruction.py:362-493``) with the reference's own
arithmetic: the ramp filter runs through ``numpy.fft`` exactly as the
reference calls it (``reconstruction.py:146-153``; complex64 forward FFT for
float32 input under NumPy >= 2, complex128 window product and inverse), one
thread per slice like the reference's joblib thread pool
(``reconstruction.py:468-475``), and the back-projection is the C
restatement of ``back_projection_cpu``.

Used by ``bench.py`` for the CPU baseline / reference arm and by tests as a
fast checker.  The product never imports it.
"""
import ctypes
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle_bp.so")
_lib = None


def build():
    """Compile ``liboracle_bp.so`` with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        lib = ctypes.CDLL(_LIB)
        lib.oracle_backproject.restype = ctypes.c_int
        lib.oracle_backproject.argtypes = [
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_int,
            ctypes.c_void_p, ctypes.c_int]
        lib.oracle_max_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def max_threads():
    return _load().oracle_max_threads()


def back_projection(sinogram, angles, center, edge_pad=False, ref_arith=True,
                    nthreads=None):
    """Back-project a 2-D [nrow, ncol] or 3-D [nrow, nslice, ncol] sinogram.

    ``ref_arith=True``: the reference's arithmetic, float32 output.
    ``ref_arith=False``: FP64 trig and accumulation, float64 output.
    """
    lib = _load()
    s = np.ascontiguousarray(sinogram, dtype=np.float32)
    two_d = s.ndim == 2
    if two_d:
        s = s[:, None, :]
    nrow, nslice, ncol = s.shape
    ang = np.ascontiguousarray(np.float32(angles))
    out = np.zeros((ncol, nslice, ncol),
                   dtype=np.float32 if ref_arith else np.float64)
    nt = nthreads or lib.oracle_max_threads()
    lib.oracle_backproject(s.ctypes.data, nrow, nslice, ncol, ang.ctypes.data,
                           float(np.float32(center)), int(bool(edge_pad)),
                           int(bool(ref_arith)), out.ctypes.data, int(nt))
    return out[:, 0, :] if two_d else out


def _ramp_window(height, width, filter_name):
    from oracle.fbp_oracle import make_2d_ramp_window
    return make_2d_ramp_window(height, width, filter_name)


def ramp_filter_ref_precision(sinogram, ramp_win, pad, pad_mode="edge"):
    """The reference's filter arithmetic: ``reconstruction.py:146-153``."""
    ncol = sinogram.shape[1]
    sp = np.pad(sinogram, ((0, 0), (pad, pad)), mode=pad_mode)
    f = np.fft.fftshift(np.fft.fft(sp), axes=1) * ramp_win
    out = np.real(np.fft.ifftshift(np.fft.ifft(np.fft.ifftshift(f, axes=1)),
                                   axes=1))
    return np.ascontiguousarray(out[:, pad:ncol + pad])


def fbp_reconstruction(sinogram, center, angles=None, ratio=1.0,
                       filter_name="hann", pad=None, pad_mode="edge",
                       nthreads=None):
    """CPU FBP of a (log) sinogram with the reference's arithmetic.

    2-D or [nrow, nslice, ncol] input, ``apply_log`` off.  Returns float32.
    """
    from oracle.fbp_oracle import make_circle_mask
    s = np.asarray(sinogram, dtype=np.float32)
    two_d = s.ndim == 2
    if two_d:
        s = s[:, None, :]
    nrow, nslice, ncol = s.shape
    if angles is None:
        angles = np.deg2rad(np.linspace(0.0, 180.0, nrow))
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    nt = nthreads or max_threads()
    win = _ramp_window(nrow, ncol + 2 * pad, filter_name)
    with ThreadPoolExecutor(max_workers=max(1, min(nt, nslice))) as ex:
        filt = list(ex.map(lambda k: ramp_filter_ref_precision(
            s[:, k, :], win, pad, pad_mode), range(nslice)))
    f = np.ascontiguousarray(np.stack(filt, axis=1), dtype=np.float32)
    rec = back_projection(f, angles, center, edge_pad=False, ref_arith=True,
                          nthreads=nt)
    if ratio is not None:
        r = ratio if ratio != 0.0 else min(center, ncol - center) / (0.5 * ncol)
        rec = rec * make_circle_mask(ncol, r)[:, None, :]
    rec = rec * np.pi / (nrow - 1)
    return rec[:, 0, :] if two_d else rec
