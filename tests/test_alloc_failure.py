"""Allocation failure through a capped allocator.

The library itself never allocates (every C entry point takes caller
buffers and workspace); the drop-in Python layer allocates through torch's
caching allocator.  Capping that allocator just above what is in use makes
the next reconstruction's allocations fail: the call must raise (no crash,
no hang, no CUDA error left behind), and once the cap is lifted the same
call must work.  The failure is made on the host, by the allocator; no
kernel faults.
"""
import numpy as np
import pytest
import torch

from algotom_b200 import _native as nat
from algotom_b200 import phantom
from algotom_b200.rec import reconstruction as R
from oracle import fbp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["fbp", "bpf"])
def test_capped_allocator_raises_and_recovers(cuda, name):
    fn = R.fbp_reconstruction if name == "fbp" else R.bpf_reconstruction
    nrow, nslice, ncol = 181, 32, 512  # each stack allocation > 10 MB
    s3 = np.stack([phantom.ellipse_sinogram(70 + k, nrow, ncol, 255.3)[0]
                   for k in range(nslice)], axis=1)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    t = torch.from_numpy(s3).to(cuda)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    total = torch.cuda.get_device_properties(cuda).total_memory
    cap = (torch.cuda.memory_reserved(cuda) + (1 << 20)) / total
    torch.cuda.set_per_process_memory_fraction(cap, cuda)
    try:
        with pytest.raises(torch.OutOfMemoryError):
            fn(t, 255.3, angles=ang, apply_log=False)
    finally:
        torch.cuda.set_per_process_memory_fraction(1.0, cuda)
    torch.cuda.synchronize()  # no CUDA error pending
    assert nat.call("atb_backproject_status", 0) == 0
    got = fn(t, 255.3, angles=ang, apply_log=False).cpu().numpy()
    ref = (O.fbp_reconstruction if name == "fbp" else O.bpf_reconstruction)(
        s3[:, 2], 255.3, angles=ang, apply_log=False)
    assert O.rel_l2(got[:, 2], ref) < 1e-5
