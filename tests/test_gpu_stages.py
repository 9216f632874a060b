"""GPU parity of the per-stage entry points (the reference's kernel free
functions) against the CPU oracle, on the golden-vector inputs and on seeded
synthetic frames.  All calls go through the C ABI of libfusion_b200.so.

Tolerances: integer, byte and index outputs exactly; float maps that the
reference-precision oracle computes with the same operation order exactly,
except the bilateral filter (CUDA's expf vs the host's expf: <= 2 ulp at 3 m,
4e-6 m); normal-equation correspondence counts exactly and sums within 2e-6
of their scale.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_util as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def S():
    from fusion_b200 import system
    return system


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _pre_inputs():
    pre = G.load("pre_128x96.npz")
    return pre, G.meta()


def test_pyramid_stages(S):
    pre, m = _pre_inputs()
    H, W = pre["depth_in"].shape
    d = dev(pre["depth_in"])
    raw = torch.empty((H, W), dtype=torch.float32, device="cuda")
    filt = torch.empty_like(raw)
    S.filter_depth(d, raw, filt, m["depth_scale"], m["depth_cutoff"])
    o_raw, o_filt = O.filter_depth(pre["depth_in"], m["depth_scale"], m["depth_cutoff"], 32)
    assert np.array_equal(host(raw), o_raw, equal_nan=True)
    f = host(filt)
    assert np.array_equal(np.isnan(f), np.isnan(o_filt))
    ok = ~np.isnan(f)
    assert np.abs(f[ok] - o_filt[ok]).max() <= 4e-6
    gray = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    S.image_to_intensity(dev(pre["rgb_in"]), gray)
    assert np.array_equal(host(gray), O.intensity(pre["rgb_in"]))
    # pyramid levels, maps and derivatives, each stage from the reference's
    # own previous-stage output so that every stage is checked on its own
    for lv in range(3):
        h, w = H >> lv, W >> lv
        s = 1 << lv
        if lv > 0:
            src_d, src_g = dev(pre[f"depth{lv - 1}"]), dev(pre[f"image{lv - 1}"])
            dd = torch.empty((h, w), dtype=torch.float32, device="cuda")
            dg = torch.empty((h, w), dtype=torch.uint8, device="cuda")
            S.pyrdown_gauss(src_d, dd)
            S.pyrdown_gauss(src_g, dg)
            od = O.pyrdown(pre[f"depth{lv - 1}"], 32)
            g_dd = host(dd)
            assert np.array_equal(np.isnan(g_dd), np.isnan(od))
            ok = ~np.isnan(od)
            assert np.array_equal(g_dd[ok], od[ok])
            assert np.array_equal(host(dg), O.pyrdown(pre[f"image{lv - 1}"], 32))
        vm = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        S.compute_vmap(dev(pre[f"depth{lv}"]), vm, m["fx"] / s, m["fy"] / s, m["cx"] / s, m["cy"] / s,
                       m["depth_cutoff"])
        ov = O.vmap(pre[f"depth{lv}"], m["fx"] / s, m["fy"] / s, m["cx"] / s, m["cy"] / s, m["depth_cutoff"], 32)
        gv = host(vm)
        val = ~np.isnan(ov[..., 0])
        assert np.array_equal(val, ~np.isnan(gv[..., 0]))
        assert np.array_equal(gv[val][:, :3], ov[val][:, :3])
        nm = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        S.compute_nmap(dev(pre[f"vmap{lv}"]), nm)
        on = O.nmap(pre[f"vmap{lv}"], 32)
        gn = host(nm)
        vn = ~np.isnan(on[..., 0])
        assert np.array_equal(vn, ~np.isnan(gn[..., 0]))
        assert np.array_equal(gn[vn], on[vn])
        dx = torch.empty((h, w), dtype=torch.int16, device="cuda")
        dy = torch.empty_like(dx)
        S.compute_derivative_image(dev(pre[f"image{lv}"]), dx, dy)
        odx, ody = O.derivative(pre[f"image{lv}"])
        assert np.array_equal(host(dx), odx) and np.array_equal(host(dy), ody)


def test_resize_map(S):
    pre, _ = _pre_inputs()
    v, n = pre["vmap0"], pre["nmap0"]
    for lv in (1, 2):
        h, w = v.shape[0] // 2, v.shape[1] // 2
        vd = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        nd = torch.empty_like(vd)
        S.resize_map(dev(v), dev(n), vd, nd)
        ov, on = O.resize_map(v, n, 32)
        gv, gn = host(vd), host(nd)
        for g, o in ((gv, ov), (gn, on)):
            val = ~np.isnan(o[..., 0])
            assert np.array_equal(val, ~np.isnan(g[..., 0]))
            assert np.array_equal(g[val], o[val])
        v, n = ov, on


@pytest.mark.parametrize("pose", ["identity", "truth"])
def test_icp_rgb_steps(S, pose):
    pre, m = _pre_inputs()
    st = G.load("steps_128x96.npz")
    Tn, Tl = st[f"pose_{pose}"], np.eye(4)
    Rc, Rci, tc = S.pose_parts(Tn)
    Rl, Rli, tl = S.pose_parts(Tl)
    for lv in range(3):
        h, w = pre[f"vmap{lv}"].shape[:2]
        s = 1 << lv
        K = np.array([m["fx"] / s, m["fy"] / s, m["cx"] / s, m["cy"] / s], np.float32)
        scratch = torch.empty(S.step_scratch_bytes(w, h), dtype=torch.uint8, device="cuda")
        res, A, b = S.icp_step(dev(st[f"B_vmap{lv}"]), dev(pre[f"vmap{lv}"]), dev(st[f"B_nmap{lv}"]),
                               dev(pre[f"nmap{lv}"]), Rc, tc, Rl, Rli, tl, K, scratch)
        So = O.icp_step(st[f"B_vmap{lv}"], pre[f"vmap{lv}"], st[f"B_nmap{lv}"], pre[f"nmap{lv}"], Tn, Tl,
                        *K.tolist(), prec=32)
        Ao, bo = O.unpack29(So)
        assert res[1] == So[28]                                  # correspondences, exact
        sc = np.abs(Ao).max()
        assert np.abs(A - Ao).max() <= 2e-6 * sc
        assert np.abs(b - bo).max() <= 2e-6 * sc
        res2, A2, b2 = S.rgb_step(dev(st[f"B_image{lv}"]), dev(pre[f"image{lv}"]), dev(st[f"B_vmap{lv}"]),
                                  dev(pre[f"vmap{lv}"]), dev(st[f"B_dx{lv}"]), dev(st[f"B_dy{lv}"]), Rc, Rci, Rl,
                                  Rli, tc, tl, K, scratch)
        So2, r2 = O.rgb_step(st[f"B_image{lv}"], pre[f"image{lv}"], st[f"B_vmap{lv}"], pre[f"vmap{lv}"],
                             st[f"B_dx{lv}"], st[f"B_dy{lv}"], Tn, Tl, *K.tolist(), prec=32)
        Ao2, bo2 = O.unpack29(So2)
        assert res2[1] == So2[28]
        sc2 = np.abs(Ao2).max()
        assert np.abs(A2 - Ao2).max() <= 2e-6 * sc2
        assert np.abs(b2 - bo2).max() <= 2e-6 * sc2


def test_bad_arguments_are_rejected(S):
    """Errors come back as status codes; nothing is launched."""
    from fusion_b200 import _lib
    L = _lib.load()
    img = _lib.Image(None, 0, 0, 0)
    assert L.fb_filter_depth(img, img, img, 5000.0, 3.0, None) == _lib.FB_EINVAL
    assert L.fb_session_create(None, None, None) == _lib.FB_EINVAL
    assert L.fb_step_scratch_bytes(0, 10) == 0
