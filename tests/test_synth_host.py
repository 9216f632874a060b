"""The seeded synthetic RGB-D generator (rgbd_synth) against its
specification, on the host: seeds are splitmix64(config << 32 | session),
sequences are deterministic, depth is u16 in 1/5000 m quantised to 1 mm,
valid depths lie in 0.3-4 m, about 2 % of them drop out to 0, the noise has
the Kinect-like sigma 0.0012 + 0.0019 (z - 0.4)^2 m, and the camera moves at
most 0.5 m/s and 30 deg/s at 30 Hz."""
import numpy as np

import rgbd_synth as synth

M64 = (1 << 64) - 1


def splitmix64(x):
    # Steele, Lea and Flood's SplitMix64 finaliser
    z = (x + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def _params(seed, **kw):
    return synth.params(160, 120, seed, fx=131.25, fy=131.25, cx=80.0, cy=60.0, depth_scale=5000.0, **kw)


def test_seeds_are_splitmix64_of_config_and_session():
    for cfg, ses in [(0, 0), (2, 0), (4, 41), (7, 123456)]:
        assert synth.session_seed(cfg, ses) == splitmix64((cfg << 32) | ses)


def test_sequences_are_deterministic_and_quantised():
    p = _params(synth.session_seed(3, 1))
    d1, c1, t1 = synth.render(p, 0, 4)
    d2, c2, t2 = synth.render(p, 0, 4)
    assert np.array_equal(d1, d2) and np.array_equal(c1, c2) and np.array_equal(t1, t2)
    v = d1[d1 > 0].astype(np.int64)
    assert v.size > 0.5 * d1.size
    assert np.all(v % 5 == 0)                               # 1 mm steps at 5000 units per metre
    assert v.min() >= 0.3 * 5000 and v.max() <= 4.0 * 5000


def test_dropouts_and_noise_model():
    seed = synth.session_seed(3, 2)
    clean, _, _ = synth.render(_params(seed, noise=0, dropout=0.0), 0, 3)
    drop, _, _ = synth.render(_params(seed, noise=0), 0, 3)
    noisy, _, _ = synth.render(_params(seed, dropout=0.0), 0, 3)
    valid = clean > 0
    lost = valid & (drop == 0)
    assert 0.01 < lost.sum() / valid.sum() < 0.03          # ~2 % dropouts
    both = valid & (noisy > 0)
    z = clean[both] / 5000.0
    e = (noisy[both].astype(np.float64) - clean[both]) / 5000.0
    tested = 0
    for lo, hi in [(0.8, 1.2), (1.2, 1.8), (1.8, 2.4), (2.4, 3.2)]:
        sel = (z >= lo) & (z < hi)
        if sel.sum() < 500:
            continue
        tested += 1
        zm = z[sel].mean()
        sigma = 0.0012 + 0.0019 * (zm - 0.4) ** 2
        assert abs(e[sel].std() / sigma - 1.0) < 0.35, (lo, hi, e[sel].std(), sigma)
        assert abs(e[sel].mean()) < 0.3 * sigma
    assert tested >= 2


def test_camera_speed_limits():
    p = _params(synth.session_seed(3, 3))
    _, _, T = synth.render(p, 0, 60, depth=False, rgb=False)
    for a, b in zip(T[:-1], T[1:]):
        assert np.linalg.norm(b[:3, 3] - a[:3, 3]) <= 0.5 / 30 + 1e-6
        R = a[:3, :3].T @ b[:3, :3]
        ang = np.degrees(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1)))
        assert ang <= 30.0 / 30 + 1e-4
