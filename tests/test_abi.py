"""The C-ABI library: it loads, exports every declared symbol, and rejects
bad arguments with error codes (no device work is started by these calls)."""
import ctypes
import os
import re

import pytest

from algotom_b200 import _native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "algotom_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(atb_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_are_exported():
    lib = nat.load()
    declared = _declared()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(nat.EXPORTS)


def test_version_and_no_error():
    assert nat.load().atb_version() >= 100
    assert isinstance(nat.last_error(), str)


def test_filter_length():
    # N itself when it is 13-smooth and cheapest: 2860 = 4 5 11 13
    assert nat.call("atb_filter_length", 2560, 150) == 2860
    # 1324 = 4 x 331 is not: the cheapest 7-smooth n >= N + ncol - 1 = 2347
    n = nat.call("atb_filter_length", 1024, 150)
    assert n >= 2347 and n <= 4096
    r = n
    for q in (2, 3, 5, 7):
        while r % q == 0:
            r //= q
    assert r == 1
    assert nat.call("atb_filter_length", 96, 14) in (124, 216, 224, 225,
                                                     240, 243, 250, 252, 256)
    rc = nat.load().atb_filter_length(20000, 150)
    assert rc == -3 and "16384" in nat.last_error()


def test_fp64_row_lengths_and_argument_errors():
    """Transform lengths of the FP64 after filter and of the autocorrelation
    metric, and their argument checks (no device work)."""
    lib = nat.load()
    assert nat.call("atb_filter_rows64_length", 2560, 150) == 2860
    assert nat.call("atb_filter_rows64_length", 61, 9) == 140  # 79 is prime
    assert nat.call("atb_autocorr_length", 2560) == 2560
    assert nat.call("atb_autocorr_length", 75) == 75
    assert nat.call("atb_autocorr_length", 61) == 125  # >= 2 x 61 - 1
    assert nat.call("atb_autocorr_length", 71) == 144
    assert lib.atb_autocorr_length(3601) == -3  # 13 x 277, 7201 > 7168
    assert lib.atb_autocorr_length(0) == -1
    one = 1
    assert lib.atb_autocorr_rowmax(None, 8, 2, 8, one, 8, one, None) == -1
    assert lib.atb_autocorr_rowmax(one, 4, 2, 8, one, 8, one, None) == -1
    rc = lib.atb_autocorr_rowmax(one, 61, 2, 61, one, 61, one, None)
    assert rc == -1 and "125" in nat.last_error()
    assert lib.atb_filter_rows64(one, 8, 2, 8, 2, 0, None, one, one, 12,
                                 None, 8, None) == -1
    rc = lib.atb_filter_rows64(one, 8, 2, 8, 2, 8, None, one, one, 12, one,
                               8, None)
    assert rc == -1 and "statistic" in nat.last_error()
    rc = lib.atb_filter_rows64(one, 8, 2, 8, 2, 0, None, one, one, 13, one,
                               8, None)
    assert rc == -1 and "12" in nat.last_error()
    assert nat.load().atb_filter_length(0, 1) == -1


def test_bad_arguments_are_rejected():
    lib = nat.load()
    # null pointers
    rc = lib.atb_backproject(None, 0, 0, 0, 10, 1, 10, None, 5.0, 0, -1.0,
                             1.0, None, 0, 0, 0, None)
    assert rc == -1 and "null" in nat.last_error()
    rc = lib.atb_filter_rows(None, 0, 0, 1, 1, 8, 0, 0, 0, None, 1, None, 4,
                             None, 0, 0, 0, None)
    assert rc == -1
    # bad shapes / enums are checked before any device work (dummy
    # non-null pointers are never dereferenced on these paths)
    p = ctypes.c_void_p(16)
    rc = lib.atb_backproject(p, 0, 0, 0, 0, 1, 10, p, 5.0, 0, -1.0, 1.0, p,
                             0, 0, 0, None)
    assert rc == -1 and "shape" in nat.last_error()
    rc = lib.atb_backproject(p, 0, 0, 0, 10, 1, 10, p, 10.0, 0, -1.0, 1.0, p,
                             0, 0, 0, None)
    assert rc == -1 and "center" in nat.last_error()
    rc = lib.atb_backproject(p, 7, 0, 0, 10, 1, 10, p, 5.0, 0, -1.0, 1.0, p,
                             0, 0, 0, None)
    assert rc == -1 and "dtype" in nat.last_error()
    rc = lib.atb_filter_rows(p, 0, 0, 4, 1, 8, 2, 42, 0, p, 1, p, 5, p, 0, 0,
                             0, None)
    assert rc == -1 and "pad_mode" in nat.last_error()
    # N = 12: 12 itself or a length >= 19 (4 and 13 are neither)
    for n in (4, 13, 18):
        rc = lib.atb_filter_rows(p, 0, 0, 4, 1, 8, 2, 0, 0, p, 1, p, n, p, 0,
                                 0, 0, None)
        assert rc == -1 and "fft_len=%d" % n in nat.last_error()
    rc = lib.atb_filter_rows(p, 0, 0, 4, 1, 8, 2, 0, 0, p, 1, p, 17, p, 0, 0,
                             0, None)  # 17 has no radix plan
    assert rc == -1 and "fft_len=17" in nat.last_error()
    rc = lib.atb_filter_rows(p, 0, 0, 4, 1, 8, 2, 0, 0, p, 3, p, 12, p, 0, 0,
                             0, None)
    assert rc == -1 and "spec_rows" in nat.last_error()


def test_call_raises_with_message():
    with pytest.raises(nat.NativeLibraryError, match="atb_filter_length"):
        nat.call("atb_filter_length", -5, 0)


def test_batch_plan_orders_by_cost():
    """The host-side work list: one unit per 64x64 tile, largest angle
    counts first, item index in the high 16 bits."""
    items = (nat.BpItem * 3)()
    for it, (nrow, ncol) in zip(items, [(100, 64), (300, 130), (200, 65)]):
        it.nrow, it.ncol = nrow, ncol
    n = nat.call("atb_bp_batch_plan", ctypes.addressof(items), 3, None, 0, 0)
    assert n == 1 + 9 + 4
    units = (ctypes.c_int * n)()
    assert nat.call("atb_bp_batch_plan", ctypes.addressof(items), 3,
                    ctypes.addressof(units), n, 0) == n
    got = [(u >> 16, u & 0xffff) for u in units]
    assert got == [(1, t) for t in range(9)] + [(2, t) for t in range(4)] + \
        [(0, 0)]
    # 32 x 32 tiles for variant 1
    assert nat.call("atb_bp_batch_plan", ctypes.addressof(items), 3, None, 0,
                    1) == 4 + 25 + 9
    lib = nat.load()
    assert lib.atb_bp_batch_plan(ctypes.addressof(items), 3,
                                 ctypes.addressof(units), 5, 0) == -3
    assert lib.atb_bp_batch_plan(ctypes.addressof(items), 3, None, 0, 2) == -1
    items[0].ncol = 20000
    assert lib.atb_bp_batch_plan(ctypes.addressof(items), 3, None, 0, 0) == -3
    assert "16384" in nat.last_error()
