"""Slice sharding across ranks, checked with 2 gloo processes on the CPU.

The reconstruction itself needs a GPU; in the gloo test each rank runs the
FP64 oracle on its slab (a stand-in with the same slab semantics), and rank
0 gathers and reassembles the stack, which must equal the unsharded result.
The GPU test runs the product's ``fbp_reconstruction`` on each of three
ranks' slabs in turn on one device and gathers them through a one-rank NCCL
group.
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


@pytest.mark.gpu
def test_device_slabs_match_whole_stack(cuda):
    """reconstruct_slab + the device fbp_reconstruction on the slabs of 3
    ranks (3, 2 and 2 of 7 slices: the 4-, 2- and 1-slice back-projection
    kernels in different mixes), gathered with gather_to_root over NCCL,
    against the whole stack in one call and against the FP64 oracle."""
    import torch.distributed as dist
    from algotom_b200 import phantom
    from algotom_b200.rec import reconstruction as REC
    from oracle import fbp_oracle as O
    nrow, nslice, ncol, cen = 181, 7, 256, 127.3
    stack = np.stack([phantom.ellipse_sinogram(70 + k, nrow, ncol, cen)[0]
                      for k in range(nslice)], axis=1).astype(np.float32)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1,
                            device_id=cuda)
    try:
        parts = [SH.reconstruct_slab(stack, cen, 3, r, REC.fbp_reconstruction,
                                     angles=ang, apply_log=False)
                 for r in range(3)]
        got = SH.gather_to_root(parts)[0]
    finally:
        dist.destroy_process_group()
    assert [(a, b) for a, b, _ in got] == [(0, 3), (3, 5), (5, 7)]
    sharded = np.concatenate([p for _, _, p in got], axis=1)
    whole = REC.fbp_reconstruction(stack, cen, angles=ang, apply_log=False)
    ref = O.fbp_reconstruction(stack, cen, angles=ang, apply_log=False)
    assert sharded.shape == whole.shape == ref.shape
    assert O.rel_l2(sharded, whole) < 1e-6
    assert O.rel_l2(sharded, ref) < 1e-5


def _oracle_partial(ratio):
    """fbp_angle_split's partial image from the FP64 oracle: ramp filter of
    the rank's rows, back-projection of its angles, the whole slice's mask
    and scale (a CPU tensor, for gloo)."""
    def fn(rows, angles, center, mask_r2, scale, ramp_win, filter_name, pad,
           pad_mode, apply_log, ncol):
        import torch
        from oracle import fbp_oracle as O
        if len(rows) == 0:
            return torch.zeros((ncol, ncol), dtype=torch.float64)
        sino = np.array(rows, dtype=np.float64)
        if apply_log:
            sino[sino <= 0.0] = 1.0
            sino = -np.log(sino)
        f = O.apply_ramp_filter(sino, None, filter_name, pad, pad_mode)
        r = O.back_projection(f, angles, center)
        mask = O._mask(ncol, center, ratio)
        return torch.from_numpy((r if mask is None else r * mask) * scale)
    return fn


def _angle_worker(rank, world, port, result_path):
    import torch.distributed as dist
    from algotom_b200 import phantom
    from oracle import fbp_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nrow, ncol, cen = 37, 40, 19.5
        sino = np.exp(-phantom.ellipse_sinogram(9, nrow, ncol, cen)[0])
        ang = np.linspace(0, np.pi, nrow, endpoint=False)
        got = SH.fbp_angle_split(sino, cen, angles=ang, ratio=0.9,
                                 partial=_oracle_partial(0.9)).numpy()
        ref = O.fbp_reconstruction(sino, cen, angles=ang, ratio=0.9)
        # the scale is the product's float32(pi) / float32(nrow - 1), the
        # oracle's pi / (nrow - 1) in FP64: 1e-7 apart
        ok = np.allclose(got, ref, rtol=0, atol=2e-7 * np.abs(ref).max())
        np.save(result_path + ".%d.npy" % rank, np.array([ok]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_angle_split_gloo(tmp_path, world):
    """fbp_angle_split on 2 and 3 gloo ranks (37 angles: uneven shares): the
    all-reduced partial images equal the whole-slice FP64 FBP on every
    rank."""
    result = str(tmp_path / "ok")
    mp.start_processes(_angle_worker, args=(world, _free_port(), result),
                       nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        assert np.load(result + ".%d.npy" % r).all()


@pytest.mark.gpu
def test_angle_split_on_device(cuda):
    """The device partial images of 3 angle shares (60 + 60 + 60 of 180
    angles) summed on one GPU, and fbp_angle_split over a one-rank NCCL
    group, against the device fbp_reconstruction of the whole slice and
    the FP64 oracle.  (Three NCCL ranks on one GPU would be kernels waiting
    on one another; the collective with more ranks is the gloo test.)"""
    import torch
    import torch.distributed as dist
    from algotom_b200 import phantom
    from algotom_b200.rec import reconstruction as REC
    from oracle import fbp_oracle as O
    nrow, ncol, cen = 180, 320, 158.6
    sino = np.exp(-phantom.ellipse_sinogram(21, nrow, ncol, cen)[0]).astype(
        np.float32)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    whole = REC.fbp_reconstruction(sino, cen, angles=ang)
    ref = O.fbp_reconstruction(sino, cen, angles=ang)
    r2, scale = REC._mask_r2(1.0, cen, ncol), REC._scale(nrow)
    acc = torch.zeros((ncol, ncol), dtype=torch.float32, device=cuda)
    for r in range(3):
        a, b = SH.slab_bounds(nrow, 3, r)
        acc += SH._device_partial(sino[a:b], ang[a:b], cen, r2, scale, None,
                                  "hann", min(int(0.15 * ncol), 150), "edge",
                                  True, ncol)
    summed = acc.cpu().numpy()
    assert O.rel_l2(summed, whole) < 1e-6
    assert O.rel_l2(summed, ref) < 1e-5
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=cuda)
    try:
        one = SH.fbp_angle_split(sino, cen, angles=ang).cpu().numpy()
    finally:
        dist.destroy_process_group()
    assert O.rel_l2(one, whole) < 1e-6
