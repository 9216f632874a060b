"""Large images: the per-stage preprocessing at 2048x2047 (just under the
2^22-pixel limit) against the reference-precision oracle, and a session at
1280x960 (twice the benchmark's size in each direction) through a few
frames: tracked, a sound map (invariant checker), vertices within the
depth range."""
import numpy as np
import pytest

import rgbd_synth as synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_preprocessing_at_the_size_limit():
    from fusion_b200 import system as S
    W, H = 2048, 2047
    p = synth.params(W, H, synth.session_seed(9, 4242), fx=525.0 * W / 640.0, fy=525.0 * W / 640.0,
                     cx=W / 2.0, cy=H / 2.0, depth_scale=5000.0)
    d, c, _ = synth.render(p, 0, 1)
    depth = d[0]
    raw = torch.empty((H, W), dtype=torch.float32, device="cuda")
    filt = torch.empty_like(raw)
    S.filter_depth(torch.from_numpy(depth).cuda(), raw, filt, 5000.0, 4.0)
    o_raw, o_filt = O.filter_depth(depth, 5000.0, 4.0, 32)
    torch.cuda.synchronize()
    assert np.array_equal(raw.cpu().numpy(), o_raw, equal_nan=True)
    f = filt.cpu().numpy()
    assert np.array_equal(np.isnan(f), np.isnan(o_filt))
    ok = ~np.isnan(f)
    assert np.abs(f[ok] - o_filt[ok]).max() <= 4e-6
    gray = torch.empty((H, W), dtype=torch.uint8, device="cuda")
    S.image_to_intensity(torch.from_numpy(c[0]).cuda(), gray)
    torch.cuda.synchronize()
    assert np.array_equal(gray.cpu().numpy(), O.intensity(c[0]))


def test_session_at_1280x960():
    from fusion_b200 import Session
    from fusion_b200.invariants import check_session
    from fusion_b200.system import make_config
    W, H = 1280, 960
    cfg = make_config(W, H, 0.008, 4, 1 << 20, 1 << 18, 1 << 18)
    p = synth.params(W, H, synth.session_seed(9, 77), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=cfg.depth_scale)
    d, c, _ = synth.render(p, 0, 4)
    s = Session(cfg)
    rs = [s.grab(d[k], c[k]) for k in range(4)]
    assert all(r.tracked for r in rs[1:])
    assert rs[-1].no_visible > 1000 and rs[-1].error_flags == 0
    assert check_session(s) == []
    lv = s.level(0, 0)
    v = lv["vmap"][..., 2]
    ok = ~np.isnan(v)
    assert ok.mean() > 0.5 and v[ok].min() > 0.1 and v[ok].max() < 4.5
    s.close()
