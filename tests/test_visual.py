"""Visual centre searches: reconstructions at candidate centres written as
TIFF files (find_center_visual_slices, algotom/rec/reconstruction.py:
1461-1533; find_center_visual_vertical_slices, algotom/rec/vertrec.py:
1431-1535).

CPU tests cover the file helpers (the next free ``Find_center_<nnn>``
folder, float TIFF writing).  GPU tests run both searches and compare the
folder and file names with those the reference wrote, and the images read
back from the files with the reference's, to 1e-5 relative L2
(``tests/golden/golden_visual.npz``).
"""
import os

import numpy as np
import pytest

from oracle import fbp_oracle as O

TOL = 1e-5
CASES = {
    "fbp_zoom": dict(start=42.0, stop=50.0, step=1.5, zoom=0.5),
    "fbp_angles": dict(start=44.0, stop=48.0, step=1.0, zoom=1.0,
                       angles=True, ratio=0.0),
    "bpf": dict(start=45.0, stop=47.0, step=0.5, zoom=1.0, method="bpf"),
    "dfi_zoom": dict(start=44.0, stop=47.0, step=1.0, zoom=0.5,
                     method="dfi", filter_name=None),
}
VCASES = {
    "after": dict(start=28.0, stop=31.0, step=1.0),
    "before_nomask": dict(start=29.0, stop=30.5, step=0.5,
                          ramp_filter="before", masking=False, alpha=30.0),
}


def _read_folder(base):
    from PIL import Image
    names = sorted(os.listdir(base))
    return names, np.stack([np.array(Image.open(os.path.join(base, n)))
                            for n in names])


# ------------------------------------------------------------- CPU
def test_folder_names(tmp_path):
    from algotom_b200.rec._files import make_folder_name
    assert make_folder_name(tmp_path, "Find_center", 3) == "Find_center_001"
    (tmp_path / "Find_center_001").mkdir()
    (tmp_path / "Find_center_003").mkdir()
    (tmp_path / "Find_center_note.txt").write_text("x")
    # three entries match the prefix: 004 is next
    assert make_folder_name(tmp_path, "Find_center", 3) == "Find_center_004"
    (tmp_path / "Find_center_004").mkdir()
    (tmp_path / "Find_center_005").mkdir()
    # five entries: 006
    assert make_folder_name(str(tmp_path), "Find_center", 3) == \
        "Find_center_006"
    assert make_folder_name(tmp_path, "Output") == "Output_00001"


def test_save_image(tmp_path):
    from PIL import Image
    from algotom_b200.rec._files import save_image
    x = np.random.default_rng(0).standard_normal((5, 7))
    p = save_image(str(tmp_path / "a" / "b" / "x.tif"), x)
    got = np.array(Image.open(p))
    assert got.dtype == np.float32 and np.array_equal(got, np.float32(x))
    p = save_image(str(tmp_path / "x.png"), x)
    got = np.array(Image.open(p))
    assert got.dtype == np.uint8 and got.max() == 255 and got.min() == 0
    with pytest.raises(ValueError, match="Can't save to tiff"):
        save_image(str(tmp_path / "c.tif"), x + 1j)


# ------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_visual_slices_match_reference(cuda, golden, tmp_path):
    from algotom_b200.rec import reconstruction as R
    g = golden("visual")
    for name, kw in CASES.items():  # in the reference run's order
        kw = dict(kw)
        if kw.get("angles") is True:
            kw["angles"] = g["angles"]
        trans = g["trans"].copy()
        base = R.find_center_visual_slices(trans, str(tmp_path), **kw)
        assert base.endswith("/")
        assert os.path.basename(base.rstrip("/")) == \
            str(g["vis__%s__folder" % name])
        names, imgs = _read_folder(base)
        assert names == list(g["vis__%s__names" % name]), name
        ref = g["vis__%s__imgs" % name]
        assert imgs.dtype == np.float32 and imgs.shape == ref.shape
        for k in range(len(names)):
            assert O.rel_l2(imgs[k], ref[k]) < TOL, (name, names[k])
        assert np.array_equal(trans, g["trans"])


@pytest.mark.gpu
def test_visual_vertical_slices_match_reference(cuda, golden, tmp_path):
    from algotom_b200.rec import vertrec as VR
    g = golden("visual")
    projs = g["cube_projs"]
    for i, (name, kw) in enumerate(VCASES.items()):
        base = VR.find_center_visual_vertical_slices(
            projs.copy(), str(tmp_path), 30, **kw, display=False)
        assert os.path.basename(base.rstrip("/")) == \
            "Find_center_%03d" % (i + 1)
        names, imgs = _read_folder(base)
        assert names == list(g["vvis__%s__names" % name]), name
        ref = g["vvis__%s__imgs" % name]
        for k in range(len(names)):
            assert O.rel_l2(imgs[k], ref[k]) < TOL, (name, names[k])


@pytest.mark.gpu
def test_reconstruct_slice_dispatch(cuda, golden):
    from algotom_b200.rec import reconstruction as R
    g = golden("visual")
    sino = -np.log(g["trans"])
    for method in ("fbp", "bpf", "dfi"):
        got = R._reconstruct_slice(sino, 46.3, method, None, 1.0, "hann",
                                   False, True, None)
        assert got.shape == (96, 96)
    with pytest.raises(NotImplementedError):
        R._reconstruct_slice(sino, 46.3, "gridrec", None, 1.0, "hann", False,
                             True, None)
