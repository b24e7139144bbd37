"""Loader for the ICRA-2020 fisheye stereo dataset layout, with the method
names of the reference's ``dataset_loader`` (Python/vfs_icra_dataset.py:30-89).

Layout under ``base_path`` (one sample per calibration file name ``<id>``):

    calib/<id>.xml                          R, t (OpenCV FileStorage nodes 'R', 't')
    image_02/data/<id>.png                  reference image (BGR)
    image_03/data/<id>.png                  other image (BGR)
    proj_depth/groundtruth/image_02/<id>.png  depth, u16, metres * 256
    result_ours/<id>depth.png               a stored result depth, same scale
    translationVector/<id>.flo              translation field (Middlebury .flo)
    calibrationVector/<id>.flo              calibration field

The dataset itself is not shipped; ``write_sample`` writes the same layout
(tests build a miniature dataset with it).  Host I/O only, no GPU work.
"""
from __future__ import annotations

import glob
import os

import numpy as np

DEPTH_SCALE = 256  # depth PNGs hold metres * 256 (Python/vfs_icra_dataset.py:37)


def _cv2():
    import cv2
    return cv2


class dataset_loader:
    """Python/vfs_icra_dataset.py:30-89."""

    def __init__(self, base_path):
        self.base_path = base_path
        self.pose_path = os.path.join(base_path, "calib")
        self.fn_xmls = sorted(glob.glob(os.path.join(self.pose_path, "*.xml")))
        self.depth_scale = DEPTH_SCALE

    def _path(self, id, folder, suffix=".png"):
        stem = os.path.splitext(os.path.basename(self.fn_xmls[id]))[0]
        return os.path.join(self.base_path, folder, stem + suffix)

    def get_calibration(self):
        """The dataset's equidistant camera: 800 px span 2*pi/3 rad of theta
        each side of the centre (400, 400), as the reference states it."""
        return 800.0 / (2 * np.pi / 3), 400, 400

    def load_pose(self, id):
        fs = _cv2().FileStorage(self.fn_xmls[id], _cv2().FileStorage_READ)
        R, t = fs.getNode("R").mat(), fs.getNode("t").mat()
        fs.release()
        return R, t

    def _depth(self, fn):
        d = _cv2().imread(fn, _cv2().IMREAD_UNCHANGED)
        if d is None:
            raise FileNotFoundError(fn)
        return (d / self.depth_scale).astype(np.float32)

    def load_depth(self, id):
        return self._depth(self._path(id, os.path.join("proj_depth", "groundtruth", "image_02")))

    def load_result(self, id):
        return self._depth(self._path(id, "result_ours", "depth.png"))

    def load_image(self, id):
        imgs = []
        for cam in ("image_02", "image_03"):
            fn = self._path(id, os.path.join(cam, "data"))
            img = _cv2().imread(fn)
            if img is None:
                raise FileNotFoundError(fn)
            imgs.append(img)
        return imgs[0], imgs[1]

    def load_vector_field(self, id):
        return (read_flo(self._path(id, "translationVector", ".flo")),
                read_flo(self._path(id, "calibrationVector", ".flo")))


# ---- Middlebury .flo: b'PIEH' (float 202021.25), int32 width, int32 height,
# then height*width*2 float32 (u, v interleaved), little endian.
_FLO_TAG = b"PIEH"


def read_flo(fn) -> np.ndarray:
    """(H, W, 2) float32 from a .flo file (what cv2.readOpticalFlow returns)."""
    with open(fn, "rb") as f:
        tag = f.read(4)
        if tag != _FLO_TAG:
            raise ValueError(f"{fn}: not a .flo file (tag {tag!r})")
        w, h = (int(v) for v in np.frombuffer(f.read(8), "<i4"))
        if w <= 0 or h <= 0:
            raise ValueError(f"{fn}: bad size {w}x{h}")
        data = np.frombuffer(f.read(4 * 2 * w * h), "<f4")
    if data.size != 2 * w * h:
        raise ValueError(f"{fn}: truncated ({data.size} of {2 * w * h} floats)")
    return data.reshape(h, w, 2).copy()


def write_flo(fn, flow) -> None:
    flow = np.asarray(flow, np.float32)
    if flow.ndim != 3 or flow.shape[2] != 2:
        raise ValueError(f"flow must be (H, W, 2), got {flow.shape}")
    h, w = flow.shape[:2]
    with open(fn, "wb") as f:
        f.write(_FLO_TAG)
        f.write(np.array([w, h], "<i4").tobytes())
        f.write(np.ascontiguousarray(flow, "<f4").tobytes())


def write_sample(base_path, name, img_ref, img_other, R, t, depth=None, tvf=None, cvf=None, result=None):
    """Write one sample in the dataset's layout (images u8 gray or BGR)."""
    cv2 = _cv2()

    def put(folder, fname, write):
        d = os.path.join(base_path, folder)
        os.makedirs(d, exist_ok=True)
        write(os.path.join(d, fname))

    def fs_write(fn):
        fs = cv2.FileStorage(fn, cv2.FileStorage_WRITE)
        fs.write("R", np.asarray(R, np.float64).reshape(3, 3))
        fs.write("t", np.asarray(t, np.float64).reshape(3, 1))
        fs.release()

    bgr = lambda a: a if a.ndim == 3 else cv2.cvtColor(a, cv2.COLOR_GRAY2BGR)
    u16 = lambda d: np.clip(np.round(np.asarray(d, np.float64) * DEPTH_SCALE), 0, 65535).astype(np.uint16)
    put("calib", name + ".xml", fs_write)
    put(os.path.join("image_02", "data"), name + ".png", lambda fn: cv2.imwrite(fn, bgr(img_ref)))
    put(os.path.join("image_03", "data"), name + ".png", lambda fn: cv2.imwrite(fn, bgr(img_other)))
    if depth is not None:
        put(os.path.join("proj_depth", "groundtruth", "image_02"), name + ".png",
            lambda fn: cv2.imwrite(fn, u16(depth)))
    if result is not None:
        put("result_ours", name + "depth.png", lambda fn: cv2.imwrite(fn, u16(result)))
    if tvf is not None:
        put("translationVector", name + ".flo", lambda fn: write_flo(fn, tvf))
    if cvf is not None:
        put("calibrationVector", name + ".flo", lambda fn: write_flo(fn, cvf))
