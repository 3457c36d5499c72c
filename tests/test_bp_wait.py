"""The back-projector's bounded staging waits, made to run out on purpose.

The TMA window staging of ``bp_kernel`` waits on an mbarrier with a poll
limit; a CTA whose wait runs out sets bit 0 of ``atb_backproject_status``
and leaves its tile unwritten rather than hang.  ``atb_backproject`` flags
bit 5 (tests only) arms the first CTA's first wait for 16 bytes more than
its copies deliver and shortens the limit to 4096 polls: every copy
completes, nothing is withheld, and the wait runs out.  The call returns
normally, the status word says so, only that tile is missing, and the
status resets.
"""
import numpy as np
import pytest
import torch

from algotom_b200 import _native as nat
from algotom_b200.rec import reconstruction as R

pytestmark = pytest.mark.gpu

TILE_X, TILE_Y = 64, 32  # pixel tile of the 4-slice CTAs


def _launch(s3, trig, ang_center, out, flags):
    nrow, nslice, ncol = s3.shape
    return nat.load().atb_backproject(
        s3.data_ptr(), nat.F32, s3.stride(0), s3.stride(1), nrow, nslice,
        ncol, trig.data_ptr(), float(np.float32(ang_center)), 0, -1.0, 1.0,
        out.data_ptr(), out.stride(0), out.stride(1), flags,
        R._stream_ptr(s3.device))


def test_staging_wait_runs_out_and_is_reported(cuda):
    rng = np.random.default_rng(5)
    nrow, nslice, ncol = 64, 4, 128   # 4-slice CTAs, 16-byte rows: TMA
    s3 = torch.from_numpy(rng.standard_normal((nrow, nslice, ncol))
                          .astype(np.float32)).cuda()
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    trig = R._trig(ang, cuda)
    nat.call("atb_backproject_status", 1)  # start clean
    ref = torch.empty((ncol, nslice, ncol), device=cuda)
    assert _launch(s3, trig, 63.3, ref, 0) == 0
    assert nat.call("atb_backproject_status", 0) == 0

    out = torch.full((ncol, nslice, ncol), float("nan"), device=cuda)
    assert _launch(s3, trig, 63.3, out, 1 << 5) == 0, nat.last_error()
    torch.cuda.synchronize()
    assert nat.call("atb_backproject_status", 0) == 1
    got, want = out.cpu().numpy(), ref.cpu().numpy()
    tile = np.zeros((ncol, nslice, ncol), bool)
    tile[:TILE_Y, :, :TILE_X] = True
    assert np.isnan(got[tile]).all()           # the stalled CTA wrote nothing
    assert np.array_equal(got[~tile], want[~tile])  # every other tile did

    assert nat.call("atb_backproject_status", 1) == 1  # read and reset
    assert nat.call("atb_backproject_status", 0) == 0
    again = torch.empty_like(ref)
    assert _launch(s3, trig, 63.3, again, 0) == 0
    assert nat.call("atb_backproject_status", 0) == 0
    assert torch.equal(again, ref)
