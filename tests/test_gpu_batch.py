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
        # same back-projection tiles; the batch filters items of similar
        # width at one shared transform length, the single-slice call at
        # its own (both exact), so the two differ by float32 rounding
        assert O.rel_l2(o, single) < 1e-6
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
    assert sum(d["half_acquisition"] for d in g1) == 8
    for k, d in enumerate(g1):
        half = k % 8 == 7
        assert d["half_acquisition"] == half
        if not half:
            assert 361 <= d["nrow"] <= 3601 and 512 <= d["ncol"] <= 4096
            assert abs(d["center"] - (d["ncol"] - 1) / 2) <= 3.0
            continue
        # 360 degrees at twice the angle count, axis 0.3 of the width
        # right of the detector centre, widened by extend_sinogram
        w, cor = d["raw_ncol"], d["raw_center"]
        assert 722 <= d["nrow"] <= 7202 and d["nrow"] % 2 == 0
        assert abs(d["angles"][1] - d["angles"][0] - 2 * np.pi / d["nrow"]) \
            < 1e-12
        assert abs(cor - ((w - 1) / 2 + 0.3 * w)) <= 3.0
        ov = int(np.round(2 * (w - cor) - 1 + 1e-3))
        assert d["ncol"] == 2 * w - ov and 1.55 * w < d["ncol"] < 1.65 * w
        assert d["center"] == w - ov / 2.0 - 0.5


def test_half_acquisition_item_reconstructs_the_object(cuda):
    """A generated 360-degree offset-axis scan, widened on the device by
    extend_sinogram and reconstructed over 360 degrees, shows the phantom
    (the generator, the extension and the batch geometry agree)."""
    w, cor, nrow = 300, 299 / 2 + 0.3 * 300, 720
    raw, ang, params, field = phantom.half_acquisition_sinogram(
        7, nrow, w, cor, photons=None)
    from algotom_b200.prep.conversion import extend_sinogram
    ext, c2 = extend_sinogram(raw, cor, apply_log=False)
    assert ext.shape[1] == field or abs(ext.shape[1] - field) <= 1
    rec = R.fbp_reconstruction(ext, c2, angles=ang, apply_log=False)
    n = ext.shape[1]
    truth = phantom.phantom_image(params, n)
    mask = O.make_circle_mask(n, 0.9)
    assert O.rel_l2(rec * mask, truth * mask) < 0.35


def test_full_uneven_batch_against_oracle(cuda):
    """The 64-item workload (widths 512-4096 and half-acquisition items
    widened to ~1.6x, 361-7202 angles) in one persistent launch: the
    narrowest and the widest item against the FP64 oracle, every item
    against the single-slice path."""
    geo = B.uneven_batch_geometry()
    sinos = B.batch_sinograms(geo, device=cuda)
    bf = B.BatchedFBP([(g["nrow"], g["ncol"]) for g in geo],
                      [g["center"] for g in geo], [g["angles"] for g in geo])
    for x, s in zip(bf.inputs, sinos):
        x.copy_(s)
    bf.capture()
    bf.replay()
    torch.cuda.synchronize()
    widths = [g["ncol"] for g in geo]
    for k in (int(np.argmin(widths)), int(np.argmax(widths))):
        g = geo[k]
        sn = sinos[k].cpu().numpy()
        f = O.apply_ramp_filter(sn, None, "hann", min(int(0.15 * g["ncol"]),
                                                      150), "edge")
        from oracle import cpu_port
        ref = cpu_port.back_projection(f.astype(np.float32), g["angles"],
                                       g["center"], ref_arith=False)
        ref = ref * O.make_circle_mask(g["ncol"], 1.0) * \
            (np.pi / (g["nrow"] - 1))
        err = O.rel_l2(bf.outputs[k].cpu().numpy(), ref)
        assert err < 1e-5, (k, g["ncol"], g["nrow"], err)
    for k in range(0, len(geo), 5):
        g = geo[k]
        single = R.fbp_reconstruction(sinos[k], g["center"],
                                      angles=g["angles"], apply_log=False)
        assert O.rel_l2(bf.outputs[k].cpu().numpy(),
                        single.cpu().numpy()) < 1e-5, k


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
