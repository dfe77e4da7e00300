import numpy as np

from word2world_b200 import camera


def test_view_matrix_convention():
    """view(x) = (right.x, -up.x, r - fwd.x) for an orbit camera at radius r
    (GaussianTrainer.py:50-83); the matrices are passed transposed."""
    cam = camera.orbit_camera(37.0, 12.0, 2.5, 256, 256)
    V = cam.viewmatrix.T.astype(np.float64)  # the math matrix
    p = np.array([0.1, -0.2, 0.3, 1.0])
    t = V @ p
    pos = -cam.campos.astype(np.float64)
    fwd = pos / np.linalg.norm(pos)
    assert abs(t[2] - (2.5 - fwd @ p[:3])) < 1e-5
    assert abs(t[3] - 1.0) < 1e-6
    # the full projection is P @ V with the perspective rows of misc_utils.get_projection_matrix
    clip = cam.projmatrix.T.astype(np.float64) @ p
    assert abs(clip[3] - t[2]) < 1e-5


def test_crop_embed_keeps_depth():
    cam = camera.orbit_camera(0.0, 0.0, 2.5, 256, 256)
    e = camera.crop_embed(cam, 800)
    assert np.array_equal(e.projmatrix[:, 2], cam.projmatrix[:, 2])
    assert np.array_equal(e.projmatrix[:, 3], cam.projmatrix[:, 3])
    p = np.array([0.05, 0.02, -0.1, 1.0], np.float64)
    c0 = cam.projmatrix.T.astype(np.float64) @ p
    c1 = e.projmatrix.T.astype(np.float64) @ p
    px0 = (c0[0] / c0[3] + 1) * 0.5 * 256 - 0.5
    px1 = (c1[0] / c1[3] + 1) * 0.5 * 800 - 0.5
    assert abs(px0 - px1) < 1e-3
