"""Key points (fb_session_set_keypoints, fb_match_descriptors) through the C ABI.

- The detector, descriptor and back-projection against their numpy
  restatement (oracle/keypoints.py) on a session's own frame: the same key
  points (positions, scales), orientations and descriptors to rounding, the
  same 3-D points and normals.  (The reference's key points come from
  OpenCV's CUDA SURF, which is not available: parity with them is unpinned.)
- The matcher against brute force in numpy.
- In a session: the bootstrap from the last frame's key points finds poses,
  keyframes are created as the camera moves and their observed keys fill the
  key map, the tracked poses stay those of the session without key points
  (the bootstrap only moves the first linearisation point), and after the
  camera is lost (frames without depth) relocalisation against the key map
  brings back the pose the session had at the same frame.
"""
import numpy as np
import pytest

import rgbd_synth as synth
from oracle import keypoints as OK
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _frames(cfg, seed, n):
    p = synth.params(cfg.width, cfg.height, seed, fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=cfg.depth_scale)
    d, c, _ = synth.render(p, 0, n)
    return d, c


def test_detector_and_backprojection_match_oracle():
    from fusion_b200 import Session, mixed_config
    cfg = mixed_config(320, 240, 0.008)
    d, c = _frames(cfg, synth.session_seed(4, 41), 1)
    s = Session(cfg)
    s.set_keypoints(True)
    s.grab(d[0], c[0])
    g = s.keypoints(0)
    lv = s.level(0, 0)
    s.close()
    # the frame's level-0 vertex and normal maps were replaced by the model
    # raycast after the key points were taken: normals again from its depth
    depth = np.ascontiguousarray(lv["depth"], np.float32)
    nm = O.nmap(O.vmap(depth, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_cutoff, 32), 32).astype(np.float32)
    kp_all, desc_all = OK.detect(lv["image"])
    kp, pts, nrm, desc = OK.backproject(kp_all, desc_all, depth, nm, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_cutoff)
    n_g, n_o = len(g["kp"]), len(kp)
    print(f"key points: {len(kp_all)} detected (oracle), {n_o} with a 3-D point (oracle) / {n_g} (GPU)")
    assert n_o > 100
    assert abs(n_g - n_o) <= 0.02 * n_o
    used, pairs = set(), []
    for i in range(n_g):
        dd = np.abs(kp[:, :2] - g["kp"][i, :2]).max(axis=1)
        j = int(np.argmin(dd))
        if dd[j] <= 1e-3 and j not in used:
            used.add(j)
            pairs.append((i, j))
    assert len(pairs) >= 0.98 * n_o
    gi, oi = np.array(pairs).T
    assert np.abs(g["kp"][gi, 2] - kp[oi, 2]).max() <= 1e-4 * kp[oi, 2].max()
    dang = np.abs(np.angle(np.exp(1j * (g["kp"][gi, 3] - kp[oi, 3]))))
    ddesc = np.abs(g["desc"][gi] - desc[oi]).max(axis=1)
    print(f"angles within 1e-3 rad: {np.mean(dang <= 1e-3):.4f}; descriptors within 1e-3: {np.mean(ddesc <= 1e-3):.4f}")
    assert np.mean(dang <= 1e-3) >= 0.97
    assert np.mean(ddesc <= 1e-3) >= 0.95
    assert np.abs(g["pts"][gi] - pts[oi]).max() <= 1e-4
    assert np.abs(g["nrm"][gi] - nrm[oi]).max() <= 1e-4
    assert np.allclose(np.linalg.norm(g["desc"], axis=1), 1.0, atol=1e-4)


def test_matcher_matches_brute_force():
    from fusion_b200.system import match_descriptors
    rng = np.random.default_rng(5)
    q = rng.normal(size=(777, 64)).astype(np.float32)
    t = rng.normal(size=(3001, 64)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    best, dist = match_descriptors(torch.from_numpy(q).cuda(), torch.from_numpy(t).cuda())
    torch.cuda.synchronize()
    ob, od = OK.match2(q, t)
    assert np.array_equal(best.cpu().numpy(), ob)
    assert np.abs(dist.cpu().numpy() - od).max() <= 1e-5


def _run(s, d, c, idx):
    rows = []
    for k in idx:
        r = s.grab(d[k], c[k])
        rows.append((r.tracked, r.tracker_state, np.array(r.pose[:]).reshape(4, 4), s.keypoint_stats()))
    return rows


def test_bootstrap_keyframes_and_relocalisation():
    from fusion_b200 import Session, mixed_config
    cfg = mixed_config(320, 240, 0.008)
    n = 24
    d, c = _frames(cfg, synth.session_seed(4, 42), n)
    plain = Session(cfg)
    base = _run(plain, d, c, range(n))
    plain.close()
    s = Session(cfg)
    s.set_keypoints(True)
    first = _run(s, d, c, range(n))
    st = s.keypoint_stats()
    boots = [r[3]["bootstrap"] for r in first[1:] if r[1] == 0]
    print(f"bootstrap found a pose on {sum(b == 1 for b in boots)} of {len(boots)} tracked frames; "
          f"{st['keyframes']} keyframes, {st['map_keys']} map keys")
    assert sum(r[0] for r in first) >= n - 2
    assert sum(b == 1 for b in boots) >= 0.8 * len(boots)
    assert st["keyframes"] >= 2 and st["map_keys"] > 50
    dmax = max(np.abs(a[2] - b[2]).max() for a, b in zip(first, base))
    print(f"poses with and without key points: max difference {dmax:.2e}")
    assert dmax <= 2e-3
    # lose the camera: frames without depth (no correspondences, no key
    # points with a 3-D point) until the tracker gives up
    d2, c2 = np.zeros_like(d[:12]), c[:12]
    lost = _run(s, d2, c2, range(12))
    print("states while blind:", [r[1] for r in lost])
    assert lost[-1][1] == -1 and not any(r[0] for r in lost)
    # back in the mapped scene: relocalisation against the key map
    back = _run(s, d, c, range(n - 8, n))
    hit = [k for k, r in enumerate(back) if r[3]["relocalised"] == 1]
    print(f"relocalised at {hit} (frames {n - 8}..{n - 1}); matches {[r[3]['matches'] for r in back]}")
    assert hit
    k = hit[0]
    T, T0 = back[k][2], first[n - 8 + k][2]
    R = T[:3, :3].T @ T0[:3, :3]
    ang = float(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1)))
    print(f"relocalised pose vs the first pass: {ang:.4f} rad, {np.abs(T[:3, 3] - T0[:3, 3]).max():.4f} m")
    assert ang <= 0.05 and np.abs(T[:3, 3] - T0[:3, 3]).max() <= 0.05
    s.close()
