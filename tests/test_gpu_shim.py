"""The C++ shim (include/fusion_b200_shim.hpp) run the way the reference's
host classes call it: oracle/_ref/shim_driver (built from
tests/shim_driver.cu against the reference's own headers by
`make -C oracle shim`) performs the reference's first-frame sequence on the
reference's DeviceArray2D buffers -- preprocessing, the pyramid, ResetMap,
FuseMapColor, CheckBlockVisibility, CreateRenderingBlocks + Raycast,
ResizeMap, ICPStep, RGBStep and RenderImage -- and every output must equal,
bit for bit, the same calls made through the C ABI directly (same library,
same inputs).  Skipped when the driver was not built (no reference sources
where the build ran)."""
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
    d, c, _ = synth.render(p, 0, 1)
    depth, rgb = np.ascontiguousarray(d[0]), np.ascontiguousarray(c[0])
    dp, cp, op = tmp_path / "depth.u16", tmp_path / "rgb.u8", tmp_path / "out.bin"
    depth.tofile(dp)
    rgb.tofile(cp)
    r = subprocess.run([DRIVER, str(W), str(H), repr(FX), repr(FY), repr(CX), repr(CY), repr(SCALE), repr(CUTOFF),
                        repr(DMIN), repr(DMAX), str(dp), str(cp), str(op)], capture_output=True, text=True,
                       timeout=300)
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
                        ("rgb_A", np.float64, 36), ("rgb_b", np.float64, 6)]:
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
