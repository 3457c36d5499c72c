"""Batched uneven FBP in one persistent launch, plain and graph-replayed."""
import numpy as np
import pytest
import torch

from algotom_b200 import phantom
from algotom_b200.rec import batch as B
from algotom_b200.rec import reconstruction as R
from oracle import fbp_oracle as O

pytestmark = pytest.mark.gpu


def _small_batch():
    geo = [(90, 64, 31.5), (181, 130, 66.0), (37, 97, 47.2), (360, 200, 98.9),
           (61, 33, 16.0), (200, 257, 130.1), (45, 321, 158.7),
           (120, 150, 73.3)]
    sinos, angs, shapes, cens = [], [], [], []
    for k, (nrow, ncol, cen) in enumerate(geo):
        s, a, _ = phantom.ellipse_sinogram(500 + k, nrow, ncol, cen,
                                           photons=1e4)
        sinos.append(s)
        angs.append(a)
        shapes.append((nrow, ncol))
        cens.append(cen)
    return sinos, angs, shapes, cens


def test_batch_matches_single_slice_and_oracle(cuda, monkeypatch):
    monkeypatch.setenv("ALGOTOM_B200_AUTOTUNE", "0")  # variant 0 both ways
    sinos, angs, shapes, cens = _small_batch()
    bf = B.BatchedFBP(shapes, cens, angs)
    outs = [o.cpu().numpy() for o in bf([torch.from_numpy(s) for s in sinos])]
    torch.cuda.synchronize()
    assert bf.counter.cpu().tolist() == [0, 0]
    for s, a, (nrow, ncol), c, o in zip(sinos, angs, shapes, cens, outs):
        single = R.fbp_reconstruction(s, c, angles=a, apply_log=False)
        assert np.array_equal(o, single)  # same tile kernel, same order
        ref = O.fbp_reconstruction(s, c, angles=a, apply_log=False)
        assert O.rel_l2(o, ref) < 1e-5


def test_batch_graph_replay(cuda):
    sinos, angs, shapes, cens = _small_batch()
    bf = B.BatchedFBP(shapes, cens, angs)
    bf([torch.from_numpy(s) for s in sinos])
    first = [o.clone() for o in bf.outputs]
    bf.capture()
    for x in bf.inputs:
        x.zero_()
    for x, s in zip(bf.inputs, sinos):
        x.copy_(torch.from_numpy(s))
    for _ in range(3):
        bf.replay()
    torch.cuda.synchronize()
    assert bf.counter.cpu().tolist() == [0, 0]
    for a, b in zip(first, bf.outputs):
        assert torch.equal(a, b)


def test_batch_limited_ctas(cuda):
    """Few CTAs each take many units; the result does not change."""
    sinos, angs, shapes, cens = _small_batch()
    bf = B.BatchedFBP(shapes, cens, angs)
    for x, s in zip(bf.inputs, sinos):
        x.copy_(torch.from_numpy(s))
    bf.launch()
    ref = [o.clone() for o in bf.outputs]
    bf.launch(max_ctas=3)
    torch.cuda.synchronize()
    for a, b in zip(ref, bf.outputs):
        assert torch.equal(a, b)


def test_uneven_geometry_is_seeded():
    g1 = B.uneven_batch_geometry()
    g2 = B.uneven_batch_geometry()
    assert [(d["nrow"], d["ncol"]) for d in g1] == \
        [(d["nrow"], d["ncol"]) for d in g2]
    assert len(g1) == 64
    assert all(361 <= d["nrow"] <= 3601 for d in g1)
    assert sum(d["half_acquisition"] for d in g1) == 8


@pytest.mark.parametrize("variant", [0, 1])
def test_batch_tile_variants(cuda, variant):
    sinos, angs, shapes, cens = _small_batch()
    bf = B.BatchedFBP(shapes, cens, angs, variant=variant)
    outs = [o.cpu().numpy() for o in bf([torch.from_numpy(s) for s in sinos])]
    for s, a, c, o in zip(sinos, angs, cens, outs):
        ref = O.fbp_reconstruction(s, c, angles=a, apply_log=False)
        assert O.rel_l2(o, ref) < 1e-5


def test_batch_autotuned(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("ALGOTOM_B200_AUTOTUNE_CACHE", str(tmp_path / "t.json"))
    sinos, angs, shapes, cens = _small_batch()
    bf = B.BatchedFBP(shapes, cens, angs)
    assert bf.variant in (0, 1)
    assert (tmp_path / "t.json").exists()
    outs = [o.cpu().numpy() for o in bf([torch.from_numpy(s) for s in sinos])]
    for s, a, c, o in zip(sinos, angs, cens, outs):
        assert O.rel_l2(o, O.fbp_reconstruction(s, c, angles=a,
                                                apply_log=False)) < 1e-5
