"""ctypes binding of ``libalgotom_b200.so`` (the C ABI in include/algotom_b200.h).

The library is built in-tree (``make -C algotom_b200/csrc`` or
``__graft_entry__.build()``) into ``algotom_b200/lib``.  There is no fallback:
if the library is missing or fails to load, every call raises
:class:`NativeLibraryError`.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libalgotom_b200.so")

# every symbol include/algotom_b200.h declares
EXPORTS = ("atb_version", "atb_last_error", "atb_copy_2d", "atb_filter_length", "atb_filter_twiddles",
           "atb_filter_rows", "atb_neg_log", "atb_backproject",
           "atb_backproject_status", "atb_backproject_centers",
           "atb_radon_workspace", "atb_radon_adjoint", "atb_bp_batch_plan",
           "atb_backproject_batch", "atb_backproject_batch_noalloc",
           "atb_gaussian_rows",
           "atb_gaussian_cols", "atb_zoom_linear", "atb_image_range",
           "atb_slice_metric_workspace", "atb_slice_metric",
           "atb_slice_entropy64", "atb_vertical_backproject",
           "atb_vertical_workspace", "atb_flat_log", "atb_shift_rows",
           "atb_extend_rows", "atb_spline_prefilter", "atb_dfi_regrid",
           "atb_bpf_filter2d_length", "atb_bpf_filter2d_workspace",
           "atb_bpf_filter2d", "atb_filter_rows_batch", "atb_shift_rows_ext",
           "atb_dfi_angle_stack", "atb_wrap_shift_rows", "atb_dfi_fft_length",
           "atb_dfi_fft_setup", "atb_dfi_rows", "atb_dfi_inverse_workspace",
           "atb_dfi_inverse", "atb_tv_workspace", "atb_tv_value",
           "atb_tv_grad", "atb_filter_rows64_length", "atb_filter_rows64",
           "atb_autocorr_length", "atb_autocorr_rowmax")

F32, F16, BF16, U16 = 0, 1, 2, 3
METRICS = {"entropy": 0, "sharpness": 1}
PAD_MODES = {"edge": 0, "constant": 1, "reflect": 2, "symmetric": 3,
             "wrap": 4, "linear_ramp": 5, "mean": 6, "maximum": 7,
             "minimum": 8, "median": 9}


class NativeLibraryError(RuntimeError):
    """The CUDA library is missing, failed to load, or a call failed."""


class FilterItem(ctypes.Structure):
    """``atb_filter_item`` of include/algotom_b200.h."""
    _fields_ = [("src", ctypes.c_void_p), ("src_row_stride", ctypes.c_int64),
                ("dst", ctypes.c_void_p), ("dst_row_stride", ctypes.c_int64),
                ("spec", ctypes.c_void_p), ("nrow", ctypes.c_int),
                ("ncol", ctypes.c_int), ("pad", ctypes.c_int),
                ("pair_offset", ctypes.c_int)]


class BpItem(ctypes.Structure):
    """``atb_bp_item`` of include/algotom_b200.h."""
    _fields_ = [("sino", ctypes.c_void_p), ("sino_row_stride", ctypes.c_int64),
                ("trig", ctypes.c_void_p), ("out", ctypes.c_void_p),
                ("out_row_stride", ctypes.c_int64), ("center", ctypes.c_double),
                ("mask_r2", ctypes.c_double), ("scale", ctypes.c_float),
                ("nrow", ctypes.c_int), ("ncol", ctypes.c_int),
                ("edge_pad", ctypes.c_int)]


_c_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_SIGS = {
    "atb_version": (ctypes.c_int, []),
    "atb_last_error": (ctypes.c_char_p, []),
    "atb_filter_length": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "atb_filter_twiddles": (ctypes.c_int, [ctypes.c_int, _vp]),
    "atb_copy_2d": (ctypes.c_int, [_vp, _c_i64, _vp, _c_i64, _c_i64, _c_i64,
                                   ctypes.c_int, _vp]),
    "atb_filter_rows": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
        ctypes.c_int, _vp, ctypes.c_int, _c_i64, _c_i64, _vp]),
    "atb_filter_rows_batch": (ctypes.c_int, [
        _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
        ctypes.c_int, ctypes.c_int, _vp]),
    "atb_neg_log": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
        _c_i64, _c_i64, _vp]),
    "atb_backproject": (ctypes.c_int, [
        _vp, ctypes.c_int, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, _vp, ctypes.c_double, ctypes.c_int, ctypes.c_double,
        ctypes.c_float, _vp, _c_i64, _c_i64, ctypes.c_int, _vp]),
    "atb_backproject_status": (ctypes.c_int, [ctypes.c_int]),
    "atb_backproject_centers": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_double,
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
        ctypes.c_float, _vp, _c_i64, _c_i64, ctypes.c_int, _vp]),
    "atb_radon_workspace": (_c_i64, [ctypes.c_int, ctypes.c_int]),
    "atb_radon_adjoint": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
        ctypes.c_double, _vp, _c_i64, _c_i64, _vp, _c_i64, _vp]),
    "atb_bp_batch_plan": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int,
                                         ctypes.c_int]),
    "atb_backproject_batch": (ctypes.c_int, [
        _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
        _vp]),
    "atb_backproject_batch_noalloc": (ctypes.c_int, [
        _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "atb_gaussian_rows": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
        _c_i64, ctypes.c_int, _vp]),
    "atb_gaussian_cols": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
        ctypes.c_int, _vp, _c_i64, _c_i64, ctypes.c_int, _vp]),
    "atb_zoom_linear": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, _vp, _c_i64, ctypes.c_int,
        ctypes.c_int, _vp]),
    "atb_image_range": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "atb_slice_metric_workspace": (_c_i64, [
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "atb_slice_metric": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, ctypes.c_float, ctypes.c_float, _vp, _c_i64, _vp,
        _vp]),
    "atb_slice_entropy64": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_double, _vp, _c_i64, _vp, _vp]),
    "atb_vertical_backproject": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp,
        ctypes.c_int, _vp, _c_i64, _c_i64, _vp, _c_i64, _vp]),
    "atb_vertical_workspace": (_c_i64, [
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "atb_shift_rows": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_double,
        ctypes.c_int, _vp, _c_i64, _vp]),
    "atb_extend_rows": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_int, ctypes.c_int, _vp, _c_i64, _vp]),
    "atb_spline_prefilter": (ctypes.c_int, [
        _vp, _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, ctypes.c_int, _vp]),
    "atb_dfi_regrid": (ctypes.c_int, [
        _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "atb_shift_rows_ext": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, _vp, _c_i64, _vp]),
    "atb_dfi_angle_stack": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, _vp, _c_i64, _c_i64, _vp]),
    "atb_wrap_shift_rows": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_int, ctypes.c_int, _vp, _c_i64, _c_i64,
        _vp]),
    "atb_dfi_fft_length": (ctypes.c_int, [ctypes.c_int]),
    "atb_tv_workspace": (_c_i64, []),
    "atb_filter_rows64_length": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "atb_filter_rows64": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        _vp, _vp, _vp, ctypes.c_int, _vp, _c_i64, _vp]),
    "atb_autocorr_length": (ctypes.c_int, [ctypes.c_int]),
    "atb_autocorr_rowmax": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp,
        _vp]),
    "atb_tv_value": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp,
        _c_i64, _vp, _vp]),
    "atb_tv_grad": (ctypes.c_int, [
        _vp, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp,
        ctypes.c_float, _vp, _c_i64, ctypes.c_int, _vp]),
    "atb_dfi_fft_setup": (ctypes.c_int, [
        ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "atb_dfi_rows": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
        _vp, _vp, _c_i64, _c_i64, _vp]),
    "atb_dfi_inverse_workspace": (_c_i64, [
        ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "atb_dfi_inverse": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp, _vp, _vp, _vp,
        _vp, _c_i64, _c_i64, ctypes.c_int, _vp, _c_i64, _vp]),
    "atb_bpf_filter2d_length": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "atb_bpf_filter2d_workspace": (_c_i64, [ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int]),
    "atb_bpf_filter2d": (ctypes.c_int, [
        _vp, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_double,
        ctypes.c_float, _vp, _c_i64, _c_i64, _vp, _c_i64, _vp]),
    "atb_flat_log": (ctypes.c_int, [
        _vp, ctypes.c_int, _c_i64, _c_i64, ctypes.c_int, ctypes.c_int,
        ctypes.c_int, _vp, _vp, _c_i64, ctypes.c_int, _vp, _c_i64, _c_i64,
        _vp, _vp]),
}

_lib = None


def load():
    """Load the library once and attach the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryError(
            "libalgotom_b200.so not built (expected at %s); run "
            "`make -C algotom_b200/csrc`" % LIB_PATH)
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as exc:
        raise NativeLibraryError("cannot load %s: %s" % (LIB_PATH, exc))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error():
    return load().atb_last_error().decode("utf-8", "replace")


def call(name, *args):
    """Call an ``atb_*`` entry point; raise on a negative return code."""
    rc = getattr(load(), name)(*args)
    if rc < 0:
        raise NativeLibraryError("%s failed (%d): %s" % (name, rc,
                                                         last_error()))
    return rc
