"""CPU tests of the data formats either side of the solve: the ICRA-2020
dataset layout (Python/vfs_icra_dataset.py:30-89), Middlebury .flo vector
fields, and the depth colour map (Python/colormap.py:286-292)."""
from __future__ import annotations

import importlib.util
import os

import numpy as np
import pytest

from helpers import pair, reference_dir

REF_COLORMAP = os.path.join(reference_dir() or os.devnull, "colormap.py")


def _sample(tmp_path, R):
    from oracle.np64 import vfs64 as V
    from vfs_b200.icra_dataset import write_sample
    p = pair(64, height=48, t=(0.1, 0.02, 0.01), seed=2)
    cam = V.EquidistantCam64(p.intrinsics)
    tvf, cvf = V.get_vector_fields(V.get_grid_zero((48, 64)) + 1, cam, cam, R, p.t, (1, 0.01))
    write_sample(str(tmp_path), "0000000042", p.img_ref, p.img_other, R, p.t, depth=p.depth, tvf=tvf, cvf=cvf,
                 result=p.depth * 0.5)
    return p, tvf.astype(np.float32), cvf.astype(np.float32)


def test_dataset_round_trip(tmp_path):
    from vfs_b200.icra_dataset import dataset_loader
    from vfs_b200.synthetic import rotation_xyz
    R = rotation_xyz(0.01, 0.02, -0.01)
    p, tvf, cvf = _sample(tmp_path, R)
    ld = dataset_loader(str(tmp_path))
    assert len(ld.fn_xmls) == 1
    f, cx, cy = ld.get_calibration()
    assert np.isclose(f, 800 / (2 * np.pi / 3)) and (cx, cy) == (400, 400)
    R2, t2 = ld.load_pose(0)
    assert np.array_equal(R2, R) and np.array_equal(t2, p.t.reshape(3, 1))
    a, b = ld.load_image(0)
    assert a.shape == (48, 64, 3) and np.array_equal(a[..., 0], p.img_ref) and np.array_equal(b[..., 2], p.img_other)
    d = ld.load_depth(0)
    z = np.clip(p.depth, 0, None)  # u16 PNGs hold no negative depths (rays beyond 90 degrees)
    assert d.dtype == np.float32 and np.abs(d - z).max() <= 0.5 / 256 + 1e-6
    assert np.abs(ld.load_result(0) - 0.5 * z).max() <= 0.5 / 256 + 1e-6
    t_, c_ = ld.load_vector_field(0)
    assert np.array_equal(t_, tvf) and np.array_equal(c_, cvf)


def test_flo_format_matches_opencv(tmp_path):
    """Our .flo writer is read by OpenCV's reader and vice versa, bit for bit."""
    import cv2
    from vfs_b200.icra_dataset import read_flo, write_flo
    rng = np.random.default_rng(1)
    flow = rng.standard_normal((7, 11, 2)).astype(np.float32)
    write_flo(tmp_path / "a.flo", flow)
    assert np.array_equal(cv2.readOpticalFlow(str(tmp_path / "a.flo")), flow)
    cv2.writeOpticalFlow(str(tmp_path / "b.flo"), flow)
    assert np.array_equal(read_flo(tmp_path / "b.flo"), flow)
    assert (tmp_path / "a.flo").read_bytes() == (tmp_path / "b.flo").read_bytes()
    (tmp_path / "c.flo").write_bytes(b"XXXX" + (tmp_path / "a.flo").read_bytes()[4:])
    with pytest.raises(ValueError):
        read_flo(tmp_path / "c.flo")
    (tmp_path / "d.flo").write_bytes((tmp_path / "a.flo").read_bytes()[:-4])
    with pytest.raises(ValueError):
        read_flo(tmp_path / "d.flo")


def test_jet_table():
    from vfs_b200.colormap import colormap, colormap_rgb
    assert colormap_rgb.shape == (256, 3)
    assert np.array_equal(colormap_rgb[0], [0, 0, 0.5156]) and np.array_equal(colormap_rgb[-1], [0.5, 0, 0])
    assert np.array_equal(colormap, colormap_rgb[:, ::-1])
    # piecewise linear ramps in 1/64 steps, each channel peaking at 1
    assert np.all(np.abs(np.diff(colormap_rgb, axis=0)) <= 1 / 64 + 1e-4)
    assert (colormap_rgb.max(0) == 1).all()


@pytest.mark.skipif(not os.path.exists(REF_COLORMAP), reason="reference checkout absent")
def test_jet_table_equals_the_reference_table():
    from vfs_b200.colormap import colormap
    spec = importlib.util.spec_from_file_location("ref_colormap", REF_COLORMAP)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert np.array_equal(colormap, mod.colormap)


def test_depth_to_colormap():
    from vfs_b200.colormap import colormap, depth_to_colormap
    d = np.array([[1.5, 10.0, 0.0], [1.0, 20.0, -1.0], [3.0, np.nan, 5.0]], np.float32)
    img = depth_to_colormap(d, 1.5, 10.0)
    assert img.shape == (3, 3, 3) and img.dtype == np.uint8
    assert np.array_equal(img[0, 0], (colormap[255] * 255).astype(np.uint8))  # near -> last entry
    assert np.array_equal(img[0, 1], (colormap[0] * 255).astype(np.uint8))    # far -> first entry
    assert np.array_equal(img[1, 0], img[0, 0]) and np.array_equal(img[1, 1], img[0, 1])  # clipped
    for y, x in ((0, 2), (1, 2), (2, 1)):
        assert not img[y, x].any()
    inv = (1 / (3.0 + 1e-6) - 0.1) / (1 / 1.5 - 0.1)
    assert np.array_equal(img[2, 0], (colormap[int(np.round(inv * 255))] * 255).astype(np.uint8))
