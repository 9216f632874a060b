"""The C++ shim (include/fusion_b200_shim.hpp) run the way the reference's
host classes call it: oracle/_ref/shim_driver (built from
tests/shim_driver.cu against the reference's own headers by
`make -C oracle shim`) performs the reference's first-frame sequence on the
reference's DeviceArray2D buffers -- preprocessing, the pyramid, ResetMap,
FuseMapColor, CheckBlockVisibility, CreateRenderingBlocks + Raycast,
ResizeMap, ICPStep, RGBStep and RenderImage -- then the mapping calls of a
second frame at a generator pose, on map buffers allocated as
Mapping::Create allocates them.  Every output must equal, bit for bit, the
same calls made through the C ABI directly (same library, same inputs),
including what the reference's callers read back from the reference's own
buffers: the visible entries (32-byte HashEntry) and counters after each
frame, the z-range images, the whole map after ExportMap (hash table, heap,
counters, the visible blocks' voxels), and an empty map after ResetMap of
the populated one.  The frame-1 z ranges are also checked against the
reference-precision oracle.  Skipped when the driver was not built (no
reference sources where the build ran)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import rgbd_synth as synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "shim_driver")
W, H = 320, 240
FX = FY = 525.0 * W / 640.0
CX, CY = W / 2.0, H / 2.0
SCALE, CUTOFF, DMIN, DMAX = 5000.0, 3.0, 0.1, 3.0


def _read(buf, off, dtype, n):
    a = np.frombuffer(buf, dtype=dtype, count=n, offset=off)
    return a, off + a.nbytes


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="shim driver not built")
def test_shim_sequence_equals_direct_calls(tmp_path):
    from fusion_b200 import _lib, system as S
    p = synth.params(W, H, synth.session_seed(5, 1), fx=FX, fy=FY, cx=CX, cy=CY, depth_scale=SCALE)
    d, c, P = synth.render(p, 0, 2)
    depth, rgb = np.ascontiguousarray(d[0]), np.ascontiguousarray(c[0])
    depth2, rgb2 = np.ascontiguousarray(d[1]), np.ascontiguousarray(c[1])
    T2 = np.linalg.inv(P[0]) @ P[1]
    dp, cp, op = tmp_path / "depth.u16", tmp_path / "rgb.u8", tmp_path / "out.bin"
    dp2, cp2, tp2 = tmp_path / "depth2.u16", tmp_path / "rgb2.u8", tmp_path / "pose2.f64"
    depth.tofile(dp)
    rgb.tofile(cp)
    depth2.tofile(dp2)
    rgb2.tofile(cp2)
    np.ascontiguousarray(T2, np.float64).tofile(tp2)
    r = subprocess.run([DRIVER, str(W), str(H), repr(FX), repr(FY), repr(CX), repr(CY), repr(SCALE), repr(CUTOFF),
                        repr(DMIN), repr(DMAX), str(dp), str(cp), str(dp2), str(cp2), str(tp2), str(op)],
                       capture_output=True, text=True, timeout=600)
    # the shim, like the reference's SafeCall, exits with status 0 on an error
    assert r.returncode == 0 and "shim driver:" in r.stdout, r.stdout + r.stderr
    buf = op.read_bytes()
    off = 0
    counts, off = _read(buf, off, np.int32, 3)
    out = {}
    n, n4, nh = W * H, W * H * 4, (W // 2) * (H // 2)
    for name, dt, k in [("raw", np.float32, n), ("filt", np.float32, n), ("gray", np.uint8, n),
                        ("vmap", np.float32, n4), ("nmap", np.float32, n4), ("depth1", np.float32, nh),
                        ("gray1", np.uint8, nh), ("dx", np.int16, n), ("dy", np.int16, n),
                        ("rvmap", np.float32, n4), ("rnmap", np.float32, n4), ("rv1", np.float32, nh * 4),
                        ("rn1", np.float32, nh * 4), ("shaded", np.uint8, n4), ("icp_res", np.float32, 2),
                        ("icp_A", np.float64, 36), ("icp_b", np.float64, 6), ("rgb_res", np.float32, 2),
                        ("rgb_A", np.float64, 36), ("rgb_b", np.float64, 6), ("more", np.int32, 10)]:
        out[name], off = _read(buf, off, dt, k)
    nvis1_dev, tiles1, fused2, visible2, rendered2, nvis2_dev, tiles2, hc, ep, visible3 = (int(x) for x in out["more"])
    n_vis1 = int(counts[1])
    NE = 1000000 + 500000          # the reference's NumEntries (fb_default_config's tables)
    NS = 700000
    for name, dt, k in [("vis1", np.int32, 8 * n_vis1), ("zx1", np.float32, 80 * 60), ("zy1", np.float32, 80 * 60),
                        ("vis2", np.int32, 8 * visible2), ("zx2", np.float32, 80 * 60),
                        ("zy2", np.float32, 80 * 60), ("table", np.int32, 8 * NE), ("heap", np.int32, NS),
                        ("vox", np.uint8, 8 * 512 * visible2), ("rv2", np.float32, n4), ("rn2", np.float32, n4),
                        ("reset", np.int32, 3)]:
        out[name], off = _read(buf, off, dt, k)
    assert off == len(buf)
    fused, visible, rendered = (int(x) for x in counts)
    print(f"shim: fused {fused} visible {visible} rendered {rendered}")
    assert fused > 100 and visible > 100 and rendered == 1

    # the same calls through the C ABI
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    emp = lambda shape, dt: torch.empty(shape, dtype=dt, device="cuda")
    raw, filt = emp((H, W), torch.float32), emp((H, W), torch.float32)
    S.filter_depth(dev(depth), raw, filt, SCALE, CUTOFF)
    gray = emp((H, W), torch.uint8)
    g_rgb = dev(rgb)
    S.image_to_intensity(g_rgb, gray)
    vmap, nmap = emp((H, W, 4), torch.float32), emp((H, W, 4), torch.float32)
    S.compute_vmap(filt, vmap, FX, FY, CX, CY, CUTOFF)
    S.compute_nmap(vmap, nmap)
    depth1, gray1 = emp((H // 2, W // 2), torch.float32), emp((H // 2, W // 2), torch.uint8)
    S.pyrdown_gauss(filt, depth1)
    S.pyrdown_gauss(gray, gray1)
    dx, dy = emp((H, W), torch.int16), emp((H, W), torch.int16)
    S.compute_derivative_image(gray, dx, dy)
    cfg = _lib.Config()
    _lib.load().fb_default_config(ctypes.byref(cfg), W, H)
    cfg.fx, cfg.fy, cfg.cx, cfg.cy = FX, FY, CX, CY
    cfg.depth_min, cfg.depth_max = DMIN, DMAX
    sess = S.Session(cfg)
    K = [FX, FY, CX, CY]
    T = np.eye(4)
    assert S.fuse_map_color(sess, raw, g_rgb, nmap, T, K) == fused
    R, Ri, t = S.pose_parts(T)
    nv = ctypes.c_uint32()
    S.check("fb_check_block_visibility", _lib.load().fb_check_block_visibility(
        sess.h, S._p(np.ascontiguousarray(R)), S._p(np.ascontiguousarray(Ri)), S._p(t), W, H,
        S._p(np.array(K, np.float32)), ctypes.byref(nv), None))
    assert nv.value == visible
    rv, rn = emp((H, W, 4), torch.float32), emp((H, W, 4), torch.float32)
    assert S.raycast(sess, rv, rn, T, K)
    rv1, rn1 = emp((H // 2, W // 2, 4), torch.float32), emp((H // 2, W // 2, 4), torch.float32)
    S.resize_map(rv, rn, rv1, rn1)
    scratch = torch.empty(S.step_scratch_bytes(W, H), dtype=torch.uint8, device="cuda")
    I3, z3 = np.eye(3, dtype=np.float32), np.zeros(3, np.float32)
    icp = S.icp_step(vmap, rv, nmap, rn, I3, z3, I3, I3, z3, K, scratch)
    rgbs = S.rgb_step(gray, gray, vmap, rv, dx, dy, I3, I3, I3, I3, z3, z3, K, scratch)
    shaded = emp((H, W, 4), torch.uint8)
    S.render_image(rv, rn, [0.0, 0.0, 0.0], shaded)
    torch.cuda.synchronize()
    L = _lib.load()
    zc, zr = (W + 7) // 8, (H + 7) // 8

    def zranges(T):
        R_, Ri_, t_ = S.pose_parts(T)
        zx, zy = emp((zr, zc), torch.float32), emp((zr, zc), torch.float32)
        nt = ctypes.c_uint32()
        S.check("fb_create_rendering_blocks", L.fb_create_rendering_blocks(
            sess.h, S._p(np.ascontiguousarray(Ri_)), S._p(t_), S._p(np.array(K, np.float32)),
            ctypes.byref(S._img(zx, 4)), ctypes.byref(S._img(zy, 4)), ctypes.byref(nt), None))
        return zx.cpu().numpy(), zy.cpu().numpy(), nt.value

    def visible_entries():
        # the visible list's order depends on the append order of the
        # visibility kernel's warps (as the reference's does): compare sorted
        e = sess.entries()[sess.visible()]
        return e[np.lexsort(e.T[::-1])]

    def rows_sorted(a):
        return a[np.lexsort(a.T[::-1])]

    # frame 1 as the reference's buffers hold it
    zx1, zy1, nt1 = zranges(T)
    assert nvis1_dev == visible and tiles1 == nt1 > 0
    v1 = out["vis1"].reshape(-1, 8)[:, :5]
    assert np.array_equal(rows_sorted(v1), visible_entries())
    assert np.array_equal(out["zx1"].reshape(60, 80)[:zr, :zc], zx1)
    assert np.array_equal(out["zy1"].reshape(60, 80)[:zr, :zc], zy1)
    # ... and the z ranges against the reference-precision oracle fed the same frame
    from oracle import oracle as O
    oc = O.config(W, H, FX, FY, CX, CY, SCALE, CUTOFF, voxel_size=cfg.voxel_size, trunc_dist=cfg.trunc_dist,
                  depth_min=DMIN, depth_max=DMAX, num_buckets=cfg.num_buckets, num_excess=cfg.num_excess,
                  num_blocks=cfg.num_blocks, precision=32)
    M = O.Map(oc)
    M.fuse(raw.cpu().numpy(), rgb, nmap.cpu().numpy(), T)
    _, _, ozmin, ozmax, otiles = M.raycast(T)
    M.close()
    assert otiles > 0
    assert np.array_equal(zx1, ozmin) and np.array_equal(zy1, ozmax)

    # frame 2 through the C ABI
    raw2, filt2 = emp((H, W), torch.float32), emp((H, W), torch.float32)
    S.filter_depth(dev(depth2), raw2, filt2, SCALE, CUTOFF)
    vmap2, nmap2 = emp((H, W, 4), torch.float32), emp((H, W, 4), torch.float32)
    S.compute_vmap(filt2, vmap2, FX, FY, CX, CY, CUTOFF)
    S.compute_nmap(vmap2, nmap2)
    assert S.fuse_map_color(sess, raw2, dev(rgb2), nmap2, T2, K) == fused2
    R2, Ri2, t2 = S.pose_parts(T2)
    S.check("fb_check_block_visibility", L.fb_check_block_visibility(
        sess.h, S._p(np.ascontiguousarray(R2)), S._p(np.ascontiguousarray(Ri2)), S._p(t2), W, H,
        S._p(np.array(K, np.float32)), ctypes.byref(nv), None))
    assert nv.value == visible2 == nvis2_dev > 100
    zx2, zy2, nt2 = zranges(T2)
    assert tiles2 == nt2 > 0 and rendered2 == 1
    v2 = out["vis2"].reshape(-1, 8)[:, :5]
    assert np.array_equal(rows_sorted(v2), visible_entries())
    assert np.array_equal(out["zx2"].reshape(60, 80)[:zr, :zc], zx2)
    assert np.array_equal(out["zy2"].reshape(60, 80)[:zr, :zc], zy2)
    rv2, rn2 = emp((H, W, 4), torch.float32), emp((H, W, 4), torch.float32)
    assert S.raycast(sess, rv2, rn2, T2, K)
    assert np.array_equal(out["rv2"].view(np.uint8), rv2.cpu().numpy().reshape(-1).view(np.uint8))
    assert np.array_equal(out["rn2"].view(np.uint8), rn2.cpu().numpy().reshape(-1).view(np.uint8))
    # the whole map exported into the reference's buffers
    e = sess.entries()
    assert np.array_equal(out["table"].reshape(-1, 8)[:, :5], e)
    st = sess.stats()
    assert (hc, ep) == (st["heap_counter"], st["entry_ptr"])
    assert np.array_equal(out["heap"], NS - 1 - np.arange(NS, dtype=np.int32))   # blocks pop from the top
    vox = np.frombuffer(out["vox"].tobytes(), dtype=[("sdf", "<f4"), ("w", "u1"), ("rgb", "u1", 3)])
    sdf_g, w_g, c_g = sess.blocks(v2[:, 3])   # the driver read the blocks in its list's order
    assert np.array_equal(vox["w"], w_g.reshape(-1))
    assert np.array_equal(vox["rgb"], c_g.reshape(-1, 3))
    assert np.array_equal(vox["sdf"].view(np.uint32), sdf_g.reshape(-1).view(np.uint32))
    # ResetMap of the populated map: the exported map is the reset state
    occupied3, hc3, ep3 = (int(x) for x in out["reset"])
    assert (occupied3, hc3, ep3, visible3) == (0, NS - 1, 1, 0)
    sess.close()

    def same(name, t):
        a, b = out[name], t.cpu().numpy().reshape(-1)
        assert a.dtype == b.dtype and a.shape == b.shape, name
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name

    for name, t in [("raw", raw), ("filt", filt), ("gray", gray), ("vmap", vmap), ("nmap", nmap),
                    ("depth1", depth1), ("gray1", gray1), ("dx", dx), ("dy", dy), ("rvmap", rv), ("rnmap", rn),
                    ("rv1", rv1), ("rn1", rn1), ("shaded", shaded)]:
        same(name, t)
    for k, (res, A, b) in (("icp", icp), ("rgb", rgbs)):
        assert np.array_equal(out[f"{k}_res"], res), k
        assert np.array_equal(out[f"{k}_A"], A.reshape(-1)), k
        assert np.array_equal(out[f"{k}_b"], b), k
    assert np.isfinite(out["icp_A"]).all() and out["icp_res"][1] > 100
