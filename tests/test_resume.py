"""Resumable slab streaming (``fbp_reconstruction(..., resume=path)``).

CPU: the manifest itself (round trip, refusal of another job's manifest,
atomic rewrite) and the argument checks.  GPU: a streamed reconstruction
interrupted after two slabs finishes, when called again, by processing only
the slabs its manifest does not list, with the same result as an
uninterrupted run.
"""
import json
import os

import numpy as np
import pytest

from algotom_b200.rec import reconstruction as R
from algotom_b200.rec.resume import SlabManifest


def test_manifest_round_trip(tmp_path):
    p = str(tmp_path / "m.json")
    key = {"shape": [10, 70, 96], "center": 47.3}
    m = SlabManifest.open(p, key)
    assert not m.is_done((0, 8)) and not os.path.exists(p)
    m.mark([(0, 8), (8, 8)])
    m.mark([(8, 8)])  # already recorded: nothing rewritten
    assert sorted(json.load(open(p))["done"]) == [[0, 8], [8, 8]]
    assert not os.path.exists(p + ".tmp")
    again = SlabManifest.open(p, key)
    assert again.is_done((0, 8)) and again.is_done((8, 8))
    assert not again.is_done((16, 16))


def test_manifest_refuses_another_job(tmp_path):
    p = str(tmp_path / "m.json")
    SlabManifest(p, {"center": 1.0}).mark([(0, 4)])
    with pytest.raises(ValueError, match="another reconstruction"):
        SlabManifest.open(p, {"center": 2.0})
    open(p, "w").write("{broken")
    with pytest.raises(ValueError, match="unreadable"):
        SlabManifest.open(p, {"center": 1.0})


def test_resume_needs_a_host_stack_and_out(tmp_path):
    s2 = np.ones((10, 32), np.float32)
    with pytest.raises(ValueError, match="resume needs"):
        R.fbp_reconstruction(s2, 15.5, apply_log=False,
                             resume=str(tmp_path / "m.json"))
    s3 = np.ones((10, 3, 32), np.float32)
    with pytest.raises(ValueError, match="resume needs"):
        R.fbp_reconstruction(s3, 15.5, apply_log=False,
                             resume=str(tmp_path / "m.json"))


@pytest.mark.gpu
def test_interrupted_stream_resumes(cuda, tmp_path, monkeypatch):
    from algotom_b200 import phantom
    nrow, nslice, ncol = 91, 70, 96
    s3 = np.stack([phantom.ellipse_sinogram(900 + k, nrow, ncol, 47.3)[0]
                   for k in range(nslice)], axis=1)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    full = R.fbp_reconstruction(s3, 47.3, angles=ang, apply_log=False)

    out = np.lib.format.open_memmap(str(tmp_path / "rec.npy"), mode="w+",
                                    dtype=np.float32,
                                    shape=(ncol, nslice, ncol))
    man = str(tmp_path / "rec.json")
    real_bp = R.backproject
    calls = {"n": 0}

    def failing(*a, **kw):
        calls["n"] += 1
        if calls["n"] == 3:
            raise RuntimeError("interrupted")
        return real_bp(*a, **kw)
    monkeypatch.setattr(R, "backproject", failing)
    with pytest.raises(RuntimeError, match="interrupted"):
        R.fbp_reconstruction(s3, 47.3, angles=ang, apply_log=False, out=out,
                             resume=man)
    done = json.load(open(man))["done"] if os.path.exists(man) else []
    assert len(done) <= 2
    spans = R._slab_spans(nslice, R.SLAB)

    calls["n"] = -10 ** 9  # no more failures; count the second run's slabs
    got = R.fbp_reconstruction(s3, 47.3, angles=ang, apply_log=False,
                               out=out, resume=man)
    assert got is out
    assert calls["n"] + 10 ** 9 == len(spans) - len(done)
    assert sorted(map(tuple, json.load(open(man))["done"])) == spans
    assert np.array_equal(np.asarray(out), full)
    # a third call finds everything done and launches nothing
    calls["n"] = 0
    R.fbp_reconstruction(s3, 47.3, angles=ang, apply_log=False, out=out,
                         resume=man)
    assert calls["n"] == 0
