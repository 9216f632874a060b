"""Staged input (fb_stage_frame): frames whose copies are started ahead and
then taken by fb_grab_frame(NULL) give the results of frames copied in by
fb_grab_frame itself, bit for bit; at most two frames wait; taking a frame
when none is staged is refused."""
import numpy as np
import pytest

import rgbd_synth as synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rows(rs):
    return [(r.tracked, r.tracker_state, r.fused, r.no_visible, r.no_allocated, tuple(r.pose[:]), r.icp_count)
            for r in rs]


def test_staged_frames_equal_direct_frames():
    from fusion_b200 import FusionError, Session, mixed_config
    cfg = mixed_config(320, 240, 0.008)
    p = synth.params(320, 240, synth.session_seed(4, 77), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=cfg.depth_scale)
    d, c, _ = synth.render(p, 0, 8)
    d = torch.from_numpy(d).pin_memory().numpy()
    c = torch.from_numpy(c).pin_memory().numpy()
    a = Session(cfg)
    direct = _rows([a.grab(d[k], c[k]) for k in range(8)])
    ea = a.entries()
    a.close()
    b = Session(cfg)
    with pytest.raises(FusionError):
        b.grab(None, None)                      # nothing staged
    b.stage(d[0], c[0])
    staged = []
    for k in range(8):
        if k + 1 < 8:
            b.stage(d[k + 1], c[k + 1])
        if k == 0:
            with pytest.raises(FusionError):
                b.stage(d[2], c[2])             # two frames wait already
        staged.append(b.grab(None, None))
    assert _rows(staged) == direct
    assert np.array_equal(b.entries(), ea)
    b.close()
