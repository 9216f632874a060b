"""Pins the CPU oracle against golden vectors produced by the reference's own
CUDA kernels (tests/golden/make_golden.py).  CPU only.

Tolerances: integer, byte and index outputs exactly; float maps within a few
float ulps (the reference build contracts some products into FMAs and uses
CUDA's expf); normal-equation sums within 1e-6 of their scale; voxels of
blocks both allocated exactly in reference precision.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_util as G

PRECS = (32, 64)


def _same_nan(a, b):
    return np.array_equal(np.isnan(a), np.isnan(b))


@pytest.fixture(scope="module")
def pre():
    return G.load("pre_128x96.npz")


@pytest.mark.parametrize("prec", PRECS)
def test_preprocess(pre, prec):
    m = G.meta()
    raw, filt = O.filter_depth(pre["depth_in"], m["depth_scale"], m["depth_cutoff"], prec)
    assert np.array_equal(raw, pre["range"], equal_nan=True)
    assert _same_nan(filt, pre["depth0"])
    ok = ~np.isnan(filt)
    assert np.abs(filt[ok] - pre["depth0"][ok]).max() <= 4e-6          # ~2 ulp at 3 m
    assert np.array_equal(O.intensity(pre["rgb_in"]), pre["image0"])
    for lv in (1, 2):
        d = O.pyrdown(pre[f"depth{lv - 1}"], prec)
        assert _same_nan(d, pre[f"depth{lv}"])
        ok = ~np.isnan(d)
        assert np.abs(d[ok] - pre[f"depth{lv}"][ok]).max() <= 4e-6
        assert np.array_equal(O.pyrdown(pre[f"image{lv - 1}"], prec), pre[f"image{lv}"])
    for lv in range(3):
        s = 1 << lv
        vm = O.vmap(pre[f"depth{lv}"], m["fx"] / s, m["fy"] / s, m["cx"] / s, m["cy"] / s,
                    m["depth_cutoff"], prec)
        r = pre[f"vmap{lv}"]
        val = ~np.isnan(r[..., 0])
        assert np.array_equal(val, ~np.isnan(vm[..., 0]))
        if prec == 32:
            assert np.array_equal(vm[val][:, :3], r[val][:, :3])
        else:
            assert np.abs(vm[val][:, :3] - r[val][:, :3]).max() <= 1e-6
        nm = O.nmap(r, prec)
        rn = pre[f"nmap{lv}"]
        vn = ~np.isnan(rn[..., 0])
        assert np.array_equal(vn, ~np.isnan(nm[..., 0]))
        assert np.abs(nm[vn] - rn[vn]).max() <= 5e-7
        dx, dy = O.derivative(pre[f"image{lv}"])
        assert np.array_equal(dx, pre[f"dx{lv}"]) and np.array_equal(dy, pre[f"dy{lv}"])


@pytest.mark.parametrize("prec", PRECS)
def test_resize_map(pre, prec):
    rs = G.load("resize_128x96.npz")
    v, n = pre["vmap0"], pre["nmap0"]
    for lv in (1, 2):
        v, n = O.resize_map(v, n, prec)
        r, rn = rs[f"vmap{lv}"], rs[f"nmap{lv}"]
        val, vn = ~np.isnan(r[..., 0]), ~np.isnan(rn[..., 0])
        assert np.array_equal(val, ~np.isnan(v[..., 0]))
        assert np.array_equal(vn, ~np.isnan(n[..., 0]))
        assert np.abs(v[val] - r[val]).max() <= 1e-6
        assert np.abs(n[vn] - rn[vn]).max() <= 3e-7
        # the four-lane normalisation quirk: |xyz| = |m| / sqrt(|m|^2 + 1) < 1
        assert np.all(np.linalg.norm(n[vn][:, :3], axis=1) < 0.75)
    v2, n2 = O.resize_map(pre["vmap0"], pre["nmap0"], prec)   # level 1 again
    assert np.isfinite(v2[~np.isnan(v2[..., 0])]).all()


def _solve(A, b):
    return np.linalg.solve(A, b)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("pose", ["identity", "truth"])
def test_icp_rgb_steps(pre, prec, pose):
    m = G.meta()
    st = G.load("steps_128x96.npz")
    Tn, Tl = st[f"pose_{pose}"], np.eye(4)
    for lv in range(3):
        s = 1 << lv
        K = (m["fx"] / s, m["fy"] / s, m["cx"] / s, m["cy"] / s)
        S = O.icp_step(st[f"B_vmap{lv}"], pre[f"vmap{lv}"], st[f"B_nmap{lv}"], pre[f"nmap{lv}"],
                       Tn, Tl, *K, prec=prec)
        A, b = O.unpack29(S)
        Ar, br, rr = st[f"icp_A_{pose}{lv}"], st[f"icp_b_{pose}{lv}"], st[f"icp_res_{pose}{lv}"]
        assert S[28] == rr[1]                                  # correspondence count, exact
        # away from the identity a pixel or two may project to a neighbouring
        # correspondence (the reference build contracts the projection into
        # FMAs): allow the products of a few rows (|row| <= ~6 here)
        scale = np.abs(Ar).max()
        assert np.abs(A - Ar).max() <= 2e-6 * scale + (0 if pose == "identity" else 2.0)
        assert np.abs(b - br).max() <= 2e-6 * scale + (0 if pose == "identity" else 0.2)
        S2, r2 = O.rgb_step(st[f"B_image{lv}"], pre[f"image{lv}"], st[f"B_vmap{lv}"], pre[f"vmap{lv}"],
                            st[f"B_dx{lv}"], st[f"B_dy{lv}"], Tn, Tl, *K, prec=prec)
        A2, b2 = O.unpack29(S2)
        Ar2, br2, rr2 = st[f"rgb_A_{pose}{lv}"], st[f"rgb_b_{pose}{lv}"], st[f"rgb_res_{pose}{lv}"]
        assert S2[28] == rr2[1] and r2[0] == rr2[1]
        scale2 = np.abs(Ar2).max()
        assert np.abs(A2 - Ar2).max() <= (2e-6 if pose == "identity" else 1e-4) * scale2
        if prec == 32:
            assert np.abs(b2 - br2).max() <= 1e-6 * np.abs(br2).max()
        # the combined Gauss-Newton step agrees to well below the pose tolerance
        x = _solve(Ar2 * 1e-4 + Ar, br2 * 1e-4 + br)
        y = _solve(A2 * 1e-4 + A, b2 * 1e-4 + b)
        assert np.abs(x - y).max() <= (1e-6 if pose == "identity" else 1e-5)


def test_hash_is_unsigned_modulo():
    """Bucket slots of the reference's head entries follow an unsigned modulo
    (NumBuckets is an unsigned constant, Mapping/DeviceMap.cu:3-10)."""
    fz = G.load("fuse_128x96.npz")
    nb = int(G.meta()["constants"]["num_buckets"])
    e, s = fz["b_entries"].astype(np.int64), fz["b_slots"]
    h = ((e[:, 0] * 73856093) & 0xFFFFFFFF) ^ ((e[:, 1] * 19349669) & 0xFFFFFFFF) ^ \
        ((e[:, 2] * 83492791) & 0xFFFFFFFF)
    head = s < nb
    assert head.sum() > 100
    assert np.array_equal(h[head] % nb, s[head])


def _fuse_check(M, fz, pfx, raw, rgb, nm, pose, prec, from_empty=True):
    nvis = M.fuse(raw, rgb, nm, pose)
    slots, ent = M.allocated()
    mine = set(map(tuple, ent[:, :3].tolist()))
    ref = set(map(tuple, fz[pfx + "entries"][:, :3].tolist()))
    # the reference drops requests under bucket-lock contention: it allocates
    # a subset of the canonical set (in reference precision)
    if prec == 32:
        assert ref <= mine
    assert len(mine ^ ref) <= 0.02 * len(ref)
    if from_empty:
        assert len(slots) == len(mine)                  # canonical insertion: no duplicates
    sdf, w, c = M.voxels(ent[:, 3])
    bi, vi = np.nonzero(w > 0)
    od = G.voxel_dict(ent, bi, vi, sdf[bi, vi], w[bi, vi], c[bi, vi])
    rd = G.voxel_dict(fz[pfx + "entries"], fz[pfx + "vox_block"], fz[pfx + "vox_index"],
                      fz[pfx + "vox_sdf"], fz[pfx + "vox_weight"], fz[pfx + "vox_rgb"])
    common = sorted(set(od) & set(rd))
    assert len(common) >= 0.98 * len(rd)
    ds = np.array([od[k][0] - rd[k][0] for k in common])
    dw = np.array([int(od[k][1]) - int(rd[k][1]) for k in common])
    dc = np.array([max(abs(a - b) for a, b in zip(od[k][2], rd[k][2])) for k in common])
    if prec == 32 and from_empty:
        # identity pose: the reference's transforms are exact, so everything is
        assert np.all(ds == 0) and np.all(dw == 0) and np.all(dc == 0)
    elif prec == 32:
        # other poses: the reference build contracts the voxel transform and
        # the colour blend into FMAs -- weights still exact, TSDF within 1e-5,
        # colours within one level
        assert np.all(dw == 0) and np.abs(ds).max() <= 1e-5 and dc.max() <= 1
    else:
        # FP64 projections land on another pixel for a few voxels
        assert np.mean(np.abs(ds) <= 1e-3) >= 0.99
        assert np.mean(dw == 0) >= 0.99 and np.mean(dc <= 1) >= 0.99
    return nvis


@pytest.mark.parametrize("prec", PRECS)
def test_fusion_from_empty_map(pre, prec):
    """Allocation + visibility + integration of frame A into an empty map,
    then frame B at the true relative pose on top of the reference's own
    state after A (teacher forcing, so the reference's dropped and duplicated
    blocks do not carry over)."""
    m = G.meta()
    fz = G.load("fuse_128x96.npz")
    st = G.load("steps_128x96.npz")
    raw_a, _ = O.filter_depth(pre["depth_in"], m["depth_scale"], m["depth_cutoff"])
    raw_b, _ = O.filter_depth(st["depth_in"], m["depth_scale"], m["depth_cutoff"])
    M = O.Map(G.oracle_config(prec))
    _fuse_check(M, fz, "a_", raw_a, pre["rgb_in"], pre["nmap0"], np.eye(4), prec)
    G.load_ref_state(M, fz, "a_")
    _fuse_check(M, fz, "b_", raw_b, st["rgb_in"], st["B_nmap0"], fz["b_pose"], prec, from_empty=False)
    M.close()


@pytest.mark.parametrize("prec", PRECS)
def test_raycast_teacher_forced(prec):
    """Raycast of the reference's own map state after frame A with its own
    visible list.  The reference's top-left 8x8 tile is blank in the golden
    run because fillBlocksKernel reads zeroed list entries past the tile count
    (Mapping/RenderScene.cu:161-175, 269); that tile is left out."""
    fz = G.load("fuse_128x96.npz")
    M = O.Map(G.oracle_config(prec))
    ent, slots = G.load_ref_state(M, fz, "a_")
    ptr2slot = dict(zip(ent[:, 3].tolist(), slots.tolist()))
    M.set_visible(np.array([ptr2slot[p] for p in fz["a_visible"][:, 3].tolist()], np.int32))
    vm, nm, zmin, zmax, tiles = M.raycast(np.eye(4))
    zr, zc = zmin.shape
    assert fz["a_zmin"][0, 0] == 0.0
    mask = np.ones(zmin.shape, bool)
    mask[0, 0] = False
    assert np.array_equal(zmin[mask], fz["a_zmin"][:zr, :zc][mask])
    assert np.array_equal(zmax, fz["a_zmax"][:zr, :zc])
    rz = fz["a_ray_vmap"]
    keep = np.ones(rz.shape[:2], bool)
    keep[:8, :8] = False
    rv, ov = ~np.isnan(rz[..., 0]) & keep, ~np.isnan(vm[..., 0]) & keep
    both = rv & ov
    assert both.sum() >= 0.998 * rv.sum() and ov.sum() <= 1.002 * rv.sum()
    d = np.abs(vm[both][:, :3] - rz[both][:, :3]).max(axis=1)
    if prec == 32:
        assert d.max() <= 1e-5
    else:
        assert np.mean(d <= 1e-4) >= 0.998
    M.close()
