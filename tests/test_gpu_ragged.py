"""Per-stage parity at ragged image sizes: widths and heights that are odd or
not multiples of 8 (the pyramid halves them with truncation, the last row
and column of every level meet the clipped filter windows), a 40x30 level
(the size at which the reference's ResizeMap bound check goes wrong), a
tiny 9x7 image, and a frame with no depth at all.  Each stage is fed the
oracle's previous-stage output and compared with the reference-precision
oracle: bit for bit, except the bilateral filter (CUDA's expf vs the host's:
4e-6 m).  All calls go through the C ABI."""
import numpy as np
import pytest

import rgbd_synth as synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SIZES = [(161, 121), (80, 60), (40, 30), (9, 7)]
SCALE, CUTOFF = 5000.0, 4.0


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _same(g, o):
    val = ~np.isnan(o[..., 0]) if o.ndim == 3 else ~np.isnan(o)
    gval = ~np.isnan(g[..., 0]) if g.ndim == 3 else ~np.isnan(g)
    assert np.array_equal(val, gval)
    assert np.array_equal(g[val], o[val])


def _frame(w, h, empty):
    p = synth.params(w, h, synth.session_seed(9, w * 1000 + h), fx=525.0 * w / 640.0, fy=525.0 * w / 640.0,
                     cx=w / 2.0, cy=h / 2.0, depth_scale=SCALE)
    d, c, _ = synth.render(p, 0, 1)
    return (np.zeros_like(d[0]) if empty else d[0]), c[0]


@pytest.mark.parametrize("empty", [False, True], ids=["scene", "no-depth"])
@pytest.mark.parametrize("size", SIZES, ids=[f"{w}x{h}" for w, h in SIZES])
def test_stages_at_ragged_sizes(size, empty):
    from fusion_b200 import system as S
    W, H = size
    depth, rgb = _frame(W, H, empty)
    fx = fy = 525.0 * W / 640.0
    cx, cy = W / 2.0, H / 2.0
    raw = torch.empty((H, W), dtype=torch.float32, device="cuda")
    filt = torch.empty_like(raw)
    S.filter_depth(dev(depth), raw, filt, SCALE, CUTOFF)
    o_raw, o_filt = O.filter_depth(depth, SCALE, CUTOFF, 32)
    assert np.array_equal(host(raw), o_raw, equal_nan=True)
    f = host(filt)
    assert np.array_equal(np.isnan(f), np.isnan(o_filt))
    ok = ~np.isnan(f)
    if ok.any():
        assert np.abs(f[ok] - o_filt[ok]).max() <= 4e-6
    gray = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    S.image_to_intensity(dev(rgb), gray)
    o_gray = O.intensity(rgb)
    assert np.array_equal(host(gray), o_gray)
    d_l, g_l = o_filt, o_gray
    v_prev = n_prev = None
    for lv in range(3):
        h, w = d_l.shape
        if h < 1 or w < 1:
            break
        s = 1 << lv
        vm = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        S.compute_vmap(dev(d_l), vm, fx / s, fy / s, cx / s, cy / s, CUTOFF)
        ov = O.vmap(d_l, fx / s, fy / s, cx / s, cy / s, CUTOFF, 32)
        gv = host(vm)
        val = ~np.isnan(ov[..., 0])
        assert np.array_equal(val, ~np.isnan(gv[..., 0]))
        assert np.array_equal(gv[val][:, :3], ov[val][:, :3])
        nm = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
        S.compute_nmap(dev(ov), nm)
        on = O.nmap(ov, 32)
        _same(host(nm), on)
        dx = torch.empty((h, w), dtype=torch.int16, device="cuda")
        dy = torch.empty_like(dx)
        S.compute_derivative_image(dev(g_l), dx, dy)
        odx, ody = O.derivative(g_l)
        assert np.array_equal(host(dx), odx) and np.array_equal(host(dy), ody)
        if v_prev is not None:
            # the raycast maps of the level above, halved (Frame::ResizeImages)
            vd = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
            nd = torch.empty_like(vd)
            S.resize_map(dev(v_prev), dev(n_prev), vd, nd)
            orv, orn = O.resize_map(v_prev, n_prev, 32)
            _same(host(vd), orv)
            _same(host(nd), orn)
        v_prev, n_prev = ov, on
        if h // 2 < 1 or w // 2 < 1:
            break
        dd = torch.empty((h // 2, w // 2), dtype=torch.float32, device="cuda")
        dg = torch.empty((h // 2, w // 2), dtype=torch.uint8, device="cuda")
        S.pyrdown_gauss(dev(d_l), dd)
        S.pyrdown_gauss(dev(g_l), dg)
        od, og = O.pyrdown(d_l, 32), O.pyrdown(g_l, 32)
        _same(host(dd), od)
        assert np.array_equal(host(dg), og)
        d_l, g_l = od, og


def test_pitched_rgb_rows():
    """RGB8 images whose rows are padded the way cudaMallocPitch pads them (a
    pitch that is a multiple of 512 bytes, not of 3): the reference's own
    DeviceArray2D<uchar3> buffers."""
    from fusion_b200 import system as S
    W, H = 320, 240
    _, rgb = _frame(W, H, False)
    padded = torch.zeros((H, 1024), dtype=torch.uint8, device="cuda")
    view = padded.as_strided((H, W, 3), (1024, 3, 1))
    view.copy_(torch.from_numpy(rgb).cuda())
    gray = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    S.image_to_intensity(view, gray)
    assert np.array_equal(host(gray), O.intensity(rgb))
