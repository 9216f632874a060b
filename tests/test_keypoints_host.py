"""Key-point host logic on the CPU: the RANSAC pose solver
(fb_pose_estimate, Solver::PoseEstimate restated) recovers a rigid motion
among outliers and is reproducible for a seed, and the numpy restatement of
the detector gives unit descriptors inside the image."""
import math

import numpy as np

import rgbd_synth as synth
from fusion_b200 import mixed_config
from fusion_b200.system import pose_estimate
from oracle import keypoints as OK
from oracle import oracle as O


def _motion(a=0.2):
    R = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    return R, np.array([0.05, -0.02, 0.03])


def test_solver_recovers_motion_among_outliers():
    rng = np.random.default_rng(0)
    ref = rng.uniform(-1, 1, (200, 3)) + [0, 0, 2]
    R, t = _motion()
    src = ref @ R.T + t + rng.normal(0, 0.003, (200, 3))
    src[:40] = rng.uniform(-1, 1, (40, 3)) + [0, 0, 2]
    ok, T, inl = pose_estimate(src, ref, 100, False, 7)
    assert ok
    assert np.abs(T[:3, :3] - R).max() < 2e-3 and np.abs(T[:3, 3] - t).max() < 3e-3
    assert inl[40:].mean() > 0.95 and inl[:40].mean() < 0.1
    ok2, T2, inl2 = pose_estimate(src, ref, 100, False, 7)
    assert ok2 and np.array_equal(T, T2) and np.array_equal(inl, inl2)


def test_solver_edge_cases():
    ok, T, _ = pose_estimate(np.zeros((2, 3)), np.zeros((2, 3)))
    assert not ok and np.array_equal(T, np.eye(4))
    # a large motion fails the motion check only while the fit is uncertain
    rng = np.random.default_rng(1)
    ref = rng.uniform(-1, 1, (50, 3)) + [0, 0, 2]
    R, t = _motion(0.6)
    ok, T, _ = pose_estimate(ref @ R.T + t, ref, 35, True, 3)
    assert ok and np.abs(T[:3, :3] - R).max() < 1e-9


def test_oracle_detector_on_a_frame():
    cfg = mixed_config(320, 240, 0.008)
    p = synth.params(320, 240, synth.session_seed(4, 41), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=5000.0)
    d, c, _ = synth.render(p, 0, 1)
    kp, desc = OK.detect(O.intensity(c[0]))
    assert 100 < len(kp) <= 320 * 240 // 100
    assert (kp[:, 0] > 0).all() and (kp[:, 0] < 320).all() and (kp[:, 1] > 0).all() and (kp[:, 1] < 240).all()
    assert np.allclose(np.linalg.norm(desc, axis=1), 1.0, atol=1e-6)
