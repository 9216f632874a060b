"""Precision form (fb_config.form = FB_FORM_PRECISION) against the FP64 oracle.

The precision form stores 6-byte voxels (FP16 TSDF, u8 weight, RGB8), fuses
in contracted FP32 and reduces the normal equations in compensated FP32 (FP64
only in the 6x6 solve).  Its results are not bit-identical to the reference's
arithmetic; this test states and bounds the errors against the FP64 oracle on
the same frames, both running free:
  - per-frame pose: rotation and translation error;
  - TSDF: RMS and maximum difference, in truncation units, over the voxels
    both maps observed; weights equal on most of them; the same block set.
The bounds are the measured values with headroom (printed by the test).
"""
import numpy as np
import pytest

import rgbd_synth as synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")


def rot_err(A, B):
    R = A[:3, :3].T @ B[:3, :3]
    return float(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1)))


def _config(form):
    from fusion_b200 import system as S
    c = S.make_config(320, 240, 0.006, 4, 1 << 18, 1 << 17, 1 << 17)
    c.form = form
    return c


def _oracle(c):
    return O.config(c.width, c.height, c.fx, c.fy, c.cx, c.cy, c.depth_scale, c.depth_cutoff,
                    voxel_size=c.voxel_size, trunc_dist=c.trunc_dist, depth_min=c.depth_min,
                    depth_max=c.depth_max, num_buckets=c.num_buckets, num_excess=c.num_excess,
                    num_blocks=c.num_blocks, iters=tuple(c.iters), precision=64)


def _observed(entries, sdf, w):
    occ = entries[:, 3] >= 0
    e = entries[occ]
    out = {}
    for b in range(len(e)):
        for v in np.nonzero(w[b] > 0)[0]:
            out[(int(e[b, 0]), int(e[b, 1]), int(e[b, 2]), int(v))] = (float(sdf[b, v]), int(w[b, v]))
    return out


def test_precision_form_errors_against_fp64_oracle():
    from fusion_b200 import Session, load
    from fusion_b200._lib import FB_FORM_PRECISION, FB_FORM_REFERENCE
    import ctypes
    n = 8
    cp = _config(FB_FORM_PRECISION)
    p = synth.params(cp.width, cp.height, synth.session_seed(9, 0), fx=cp.fx, fy=cp.fy, cx=cp.cx, cy=cp.cy,
                     depth_scale=cp.depth_scale)
    depth, rgb, _ = synth.render(p, 0, n)
    lib = load()
    saved = lib.fb_session_bytes(ctypes.byref(_config(FB_FORM_REFERENCE))) - lib.fb_session_bytes(ctypes.byref(cp))
    assert saved == 2 * 512 * cp.num_blocks                      # 8 -> 6 bytes per voxel
    s = Session(cp)
    sysm = O.System(_oracle(cp))
    rot, tra = [], []
    for k in range(n):
        r = s.grab(depth[k], rgb[k])
        info = sysm.grab(depth[k], rgb[k])
        assert r.tracked == int(info[0])
        Pg = np.array(r.pose[:]).reshape(4, 4)
        Po = sysm.pose(0)
        rot.append(rot_err(Pg, Po))
        tra.append(float(np.abs(Pg[:3, 3] - Po[:3, 3]).max()))
    # maps: voxels observed by both
    e_g = s.entries()
    occ = e_g[:, 3] >= 0
    sdf_g, w_g, _ = s.blocks(e_g[occ][:, 3])
    e_o = sysm.map.entries()
    occ_o = e_o[:, 3] >= 0
    sdf_o, w_o, _ = sysm.map.voxels(e_o[occ_o][:, 3])
    vg = _observed(e_g, sdf_g, w_g)
    vo = _observed(e_o, sdf_o, w_o)
    common = vg.keys() & vo.keys()
    d = np.array([vg[k][0] - vo[k][0] for k in common])
    eq = np.array([vg[k][1] == vo[k][1] for k in common])
    same_w = eq.mean()
    rms_eq = float(np.sqrt(np.mean(d[eq] ** 2)))
    blocks_g = {tuple(x[:3]) for x in e_g[occ]}
    blocks_o = {tuple(x[:3]) for x in e_o[occ_o]}
    print(f"precision form vs FP64 oracle, free running: max rot {max(rot):.2e} rad, max t {max(tra):.2e} m, "
          f"TSDF rms {np.sqrt(np.mean(d ** 2)):.2e} max {np.abs(d).max():.2e} (truncation units), "
          f"rms where weights agree {rms_eq:.2e}, weights equal {same_w:.4f}, voxels {len(common)} of {len(vo)}, "
          f"blocks {len(blocks_g & blocks_o)} common / {len(blocks_o)} oracle / {len(blocks_g)} gpu")
    # free running, the TSDF difference includes the poses' (a 5e-5 m camera
    # offset is 2e-3 of a 24 mm truncation): the storage and arithmetic error
    # alone is the teacher-forced test below
    assert max(rot) <= 2e-3 and max(tra) <= 2e-3
    assert np.sqrt(np.mean(d ** 2)) <= 1e-2
    assert len(common) >= 0.95 * len(vo)
    assert same_w >= 0.95
    assert len(blocks_g ^ blocks_o) <= 0.02 * len(blocks_o)
    s.close()
    sysm.close()


def test_precision_form_in_a_batch_equals_it_alone():
    from fusion_b200 import Batch, Session
    from fusion_b200._lib import FB_FORM_PRECISION
    c = _config(FB_FORM_PRECISION)
    p = synth.params(c.width, c.height, synth.session_seed(9, 1), fx=c.fx, fy=c.fy, cx=c.cx, cy=c.cy,
                     depth_scale=c.depth_scale)
    depth, rgb, _ = synth.render(p, 0, 5)
    a = Session(c)
    alone = [tuple(a.grab(depth[k], rgb[k]).pose[:]) for k in range(5)]
    e_a = a.entries()
    a.close()
    s1, s2 = Session(c), Session(c)
    with Batch() as b:
        both = [b.step([s1, s2], [(depth[k], rgb[k]), (depth[k], rgb[k])]) for k in range(5)]
    assert [tuple(r[0].pose[:]) for r in both] == alone
    assert [tuple(r[1].pose[:]) for r in both] == alone
    assert np.array_equal(s1.entries(), e_a)
    s1.close()
    s2.close()


def test_precision_form_integration_teacher_forced():
    """Integration alone: the same raw depth, colour, normals and poses (the
    generator's true poses) fused into a precision-form session and into the
    FP64 oracle's map; the TSDF difference is then FP16 storage plus FP32
    arithmetic (and the rare voxel whose projection lands on the other side
    of a pixel boundary)."""
    import torch
    from fusion_b200 import Session
    from fusion_b200 import system as S
    from fusion_b200._lib import FB_FORM_PRECISION
    c = _config(FB_FORM_PRECISION)
    p = synth.params(c.width, c.height, synth.session_seed(9, 2), fx=c.fx, fy=c.fy, cx=c.cx, cy=c.cy,
                     depth_scale=c.depth_scale)
    depth, rgb, poses = synth.render(p, 0, 3)
    s = Session(c)
    M = O.Map(_oracle(c))
    K = np.array([c.fx, c.fy, c.cx, c.cy], np.float32)
    for k in range(3):
        raw, filt = O.filter_depth(depth[k], c.depth_scale, c.depth_cutoff, 64)
        vm = O.vmap(filt.astype(np.float32), c.fx, c.fy, c.cx, c.cy, c.depth_cutoff, 64)
        nm = O.nmap(vm, 64).astype(np.float32)
        raw32 = raw.astype(np.float32)
        n_o = M.fuse(raw32, rgb[k], nm, poses[k])
        n_g = S.fuse_map_color(s, torch.from_numpy(raw32).cuda(), torch.from_numpy(np.ascontiguousarray(rgb[k])).cuda(),
                               torch.from_numpy(nm).cuda(), poses[k], K)
        assert abs(n_g - n_o) <= 0.005 * n_o
    e_g = s.entries()
    occ = e_g[:, 3] >= 0
    sdf_g, w_g, c_g = s.blocks(e_g[occ][:, 3])
    e_o = M.entries()
    occ_o = e_o[:, 3] >= 0
    sdf_o, w_o, c_o = M.voxels(e_o[occ_o][:, 3])
    bg, bo = {tuple(x[:3]) for x in e_g[occ]}, {tuple(x[:3]) for x in e_o[occ_o]}
    assert len(bg ^ bo) <= 0.005 * len(bo)      # allocation decisions in FP32 vs FP64
    vg, vo = _observed(e_g, sdf_g, w_g), _observed(e_o, sdf_o, w_o)
    common = vg.keys() & vo.keys()
    d = np.array([vg[k][0] - vo[k][0] for k in common])
    eq = np.array([vg[k][1] == vo[k][1] for k in common])
    rms, rms_eq = float(np.sqrt(np.mean(d ** 2))), float(np.sqrt(np.mean(d[eq] ** 2)))
    # colours of the voxels both observed: the blend c0 + 0.2 w (c - c0) in
    # FP32 floors where the reference truncates toward zero (they differ
    # where the sum is negative and wraps), so a colour may be one level off
    # per observation
    def colours(e, occ_, c, w):
        rows = e[occ_]
        out = {}
        for b in range(len(rows)):
            for v in np.nonzero(w[b] > 0)[0]:
                out[(int(rows[b, 0]), int(rows[b, 1]), int(rows[b, 2]), int(v))] = c[b, v].astype(int)
        return out
    cg_, co_ = colours(e_g, occ, c_g, w_g), colours(e_o, occ_o, c_o, w_o)
    dc = np.array([np.abs(cg_[k] - co_[k]).max() for k in common])
    within1 = float(np.mean(dc <= 1))
    print(f"precision form integration vs FP64 oracle, same inputs: TSDF rms {rms:.2e}, rms where weights "
          f"agree {rms_eq:.2e}, max {np.abs(d).max():.2e} (truncation units); weights equal {eq.mean():.5f}; "
          f"colours equal {np.mean(dc == 0):.4f}, within 1 level {within1:.4f}; "
          f"voxels {len(common)} of {len(vo)} oracle / {len(vg)} gpu")
    assert within1 >= 0.99
    assert rms_eq <= 1e-3            # FP16 storage: half an ulp is 2.4e-4 at |sdf| in [0.5, 1)
    assert eq.mean() >= 0.999
    assert len(common) >= 0.999 * len(vo)
    s.close()
    M.close()
