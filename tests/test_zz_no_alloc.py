"""The allocation-free batch entry point against the allocating one.

atb_backproject_batch_noalloc serves callers that hold device buffers for
their data but may not call cudaMalloc (e.g. a plugin whose host application
owns the device memory budget).  It keeps its scratch in a fixed device
array of the library.  This test drives it through the C ABI, twice in a
row (the second call, with a smaller table, must not run the first call's
leftover entries), and compares its output with atb_backproject_batch, which
takes caller-allocated scratch.
The file name keeps it last in collection order.
"""
import ctypes

import numpy as np
import pytest
import torch

from algotom_b200 import _native as nat
from algotom_b200 import phantom
from algotom_b200.rec import batch as B
from algotom_b200.rec import reconstruction as R
from oracle import fbp_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, the bar every FP32 reconstruction is held to


def _batch():
    geo = [(90, 64, 31.5), (181, 130, 66.0), (37, 97, 47.2), (240, 200, 98.9),
           (61, 33, 16.0), (120, 257, 130.1)]
    sinos, angs, shapes, cens = [], [], [], []
    for k, (nrow, ncol, cen) in enumerate(geo):
        s, a, _ = phantom.ellipse_sinogram(900 + k, nrow, ncol, cen,
                                           photons=1e4)
        sinos.append(s)
        angs.append(a)
        shapes.append((nrow, ncol))
        cens.append(cen)
    return sinos, angs, shapes, cens


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    sinos, angs, shapes, cens = _batch()
    bf = B.BatchedFBP(shapes, cens, angs)
    for x, s in zip(bf.inputs, sinos):
        x.copy_(torch.from_numpy(s))
    bf.launch()  # filter + atb_backproject_batch (caller-provided scratch)
    torch.cuda.synchronize()
    reference = [o.clone() for o in bf.outputs]
    stream = R._stream_ptr(cuda)
    lib = nat.load()

    # first call: the whole 6-item table
    for o in bf.outputs:
        o.fill_(float("nan"))
    table = (nat.BpItem * bf.n)()
    ctypes.memmove(table, bf.items_host, ctypes.sizeof(table))
    rc = lib.atb_backproject_batch_noalloc(ctypes.addressof(table), bf.n, 0,
                                           stream)
    assert rc == 0, nat.last_error()
    # the host table is the caller's again once the call has returned
    ctypes.memset(table, 0, ctypes.sizeof(table))
    torch.cuda.synchronize()
    for ref, got in zip(reference, bf.outputs):
        assert torch.isfinite(got).all()
        assert O.rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < TOL
    oracle = O.fbp_reconstruction(sinos[0], cens[0], angles=angs[0],
                                  apply_log=False)
    assert O.rel_l2(bf.outputs[0].cpu().numpy(), oracle) < TOL

    # second call: a smaller, different table (items 4 and 1, in that
    # order); the first call's six entries are still in the shared array,
    # and none of them may be run again
    for o in bf.outputs:
        o.fill_(float("nan"))
    pick = [4, 1]
    small = (nat.BpItem * len(pick))()
    for k, b in enumerate(pick):
        ctypes.memmove(ctypes.addressof(small) + k * ctypes.sizeof(nat.BpItem),
                       ctypes.addressof(bf.items_host)
                       + b * ctypes.sizeof(nat.BpItem),
                       ctypes.sizeof(nat.BpItem))
    rc = lib.atb_backproject_batch_noalloc(ctypes.addressof(small), len(pick),
                                           0, stream)
    assert rc == 0, nat.last_error()
    torch.cuda.synchronize()
    for b, (ref, got) in enumerate(zip(reference, bf.outputs)):
        if b in pick:
            assert torch.isfinite(got).all(), b
            assert O.rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < TOL, b
        else:
            assert torch.isnan(got).all(), b
    oracle = O.fbp_reconstruction(sinos[1], cens[1], angles=angs[1],
                                  apply_log=False)
    assert O.rel_l2(bf.outputs[1].cpu().numpy(), oracle) < TOL


def test_noalloc_rejects_oversized_batches(cuda):
    items = (nat.BpItem * 4097)()
    lib = nat.load()
    rc = lib.atb_backproject_batch_noalloc(ctypes.addressof(items), 4097, 0,
                                           None)
    assert rc == -3 and "4096" in nat.last_error()
    one = (nat.BpItem * 1)()
    t = torch.zeros(1, device=cuda)
    one[0].sino = one[0].trig = one[0].out = t.data_ptr()
    one[0].nrow, one[0].ncol, one[0].center = 10, 20000, 5.0
    rc = lib.atb_backproject_batch_noalloc(ctypes.addressof(one), 1, 0, None)
    assert rc == -3 and "16384" in nat.last_error()
    one[0].ncol = 16384  # 256 x 256 tiles: within the 1048576-tile limit
    big = (nat.BpItem * 17)()
    for it in big:
        it.sino = it.trig = it.out = t.data_ptr()
        it.nrow, it.ncol, it.center = 10, 16384, 5.0
    rc = lib.atb_backproject_batch_noalloc(ctypes.addressof(big), 17, 0, None)
    assert rc == -3 and "1048576" in nat.last_error()
