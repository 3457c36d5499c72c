"""Slice sharding across ranks, checked with 2 gloo processes on the CPU.

The reconstruction itself needs a GPU; here each rank runs the FP64 oracle
on its slab (a stand-in with the same slab semantics), and rank 0 gathers
and reassembles the stack, which must equal the unsharded result.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from algotom_b200.rec import sharding as SH


def test_slab_bounds_cover_exactly():
    for nslice in (1, 7, 256, 257):
        for world in (1, 2, 3, 8):
            spans = [SH.slab_bounds(nslice, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nslice
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        SH.slab_bounds(10, 2, 2)


def test_lpt_assign_balances_and_is_deterministic():
    rng = np.random.default_rng(0)
    shapes = [(int(rng.integers(361, 3602)), int(rng.integers(512, 4097)))
              for _ in range(64)]
    costs = SH.item_costs(shapes)
    a = SH.lpt_assign(costs, 8)
    assert a == SH.lpt_assign(costs, 8)
    assert sorted(i for part in a for i in part) == list(range(64))
    loads = [sum(costs[i] for i in part) for part in a]
    # LPT bound: max load <= 4/3 of the optimum (>= mean)
    assert max(loads) <= 4.0 / 3.0 * max(np.mean(loads), max(costs)) + 1e-6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_path):
    import torch.distributed as dist
    from algotom_b200 import phantom
    from oracle import fbp_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nrow, nslice, ncol = 24, 5, 32
        stack = np.stack([phantom.ellipse_sinogram(40 + k, nrow, ncol,
                                                   15.5)[0]
                          for k in range(nslice)], axis=1)
        ang = np.linspace(0, np.pi, nrow, endpoint=False)
        start, stop, part = SH.reconstruct_slab(
            stack, 15.5, world, rank, O.fbp_reconstruction, angles=ang,
            apply_log=False)
        got = SH.gather_to_root((start, stop, part))
        if rank == 0:
            full = np.concatenate([p for _, _, p in sorted(
                got, key=lambda t: t[0])], axis=1)
            ref = O.fbp_reconstruction(stack, 15.5, angles=ang,
                                       apply_log=False)
            np.save(result_path, np.array([full.shape == ref.shape,
                                           np.array_equal(full, ref)]))
    finally:
        dist.destroy_process_group()


def test_two_rank_slab_sharding_gloo(tmp_path):
    result = str(tmp_path / "ok.npy")
    mp.start_processes(_worker, args=(2, _free_port(), result), nprocs=2,
                       join=True, start_method="spawn")
    ok = np.load(result)
    assert ok.all()
