"""The reference's vector-field test (Python/test_vector_field.py:36-66) through
the dataset loader: fields stored in the ICRA-2020 layout are read back and
compared with the CUDA generator at the reference test's bound (5e-4 px).

The dataset is not shipped, so the stored fields come from the float64
oracle, written into a miniature dataset at the dataset's own geometry
(800x800, dataset_loader.get_calibration()) with a rotated, translated pose.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_vector_fields_against_stored_dataset_fields(gpu, tmp_path):
    from oracle.np64 import vfs64 as V
    from vfs_b200 import EquidistantCam
    from vfs_b200.icra_dataset import dataset_loader, write_sample
    from vfs_b200.synthetic import rotation_xyz
    from vfs_b200.vector_field import get_grid_one, get_vector_fields
    h = w = 800
    R = rotation_xyz(0.004, -0.012, 0.003)
    t = np.array([[0.3], [0.01], [-0.02]])
    f, cx, cy = dataset_loader(str(tmp_path)).get_calibration()
    cam64 = V.EquidistantCam64((f, cx, cy))
    tvf, cvf = V.get_vector_fields(V.get_grid_zero((h, w)) + 1, cam64, cam64, R, t, (1, 0.01))
    img = np.zeros((h, w), np.uint8)
    write_sample(str(tmp_path), "0000000103", img, img, R, t, tvf=tvf, cvf=cvf)

    loader = dataset_loader(str(tmp_path))
    cam = EquidistantCam(loader.get_calibration())
    cam.setup_module()
    R2, t2 = loader.load_pose(0)
    tvf_ref, cvf_ref = loader.load_vector_field(0)
    got_t, got_c = get_vector_fields(get_grid_one((h, w)), cam, cam, R2, t2, (1, 0.01))
    got_t, got_c = np.asarray(got_t), np.asarray(got_c)
    ok = np.isfinite(tvf_ref).all(-1)  # the field is undefined at the epipoles
    assert ok.mean() > 0.999
    assert np.max(np.abs(tvf_ref - got_t)[ok]) < 5e-4
    assert np.max(np.abs(cvf_ref - got_c)) < 5e-4
