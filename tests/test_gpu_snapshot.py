"""Session snapshots (fb_snapshot / fb_restore) through the C ABI: a session
restored from a snapshot continues exactly as the original does -- every
later frame's pose and counts and the final hash table and voxels are the
same bits -- in both voxel forms; a snapshot is refused by a session of
another configuration."""
import hashlib

import numpy as np
import pytest

import rgbd_synth as synth

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")


def _digest(sess):
    e = sess.entries()
    occ = e[:, 3] >= 0
    sdf, w, c = sess.blocks(e[occ][:, 3])
    h = hashlib.sha1()
    for a in (e, sdf.view(np.uint32), w, c):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _row(r):
    return (r.tracked, r.tracker_state, r.fused, r.no_visible, r.no_allocated, r.no_new, tuple(r.pose[:]))


@pytest.mark.parametrize("form", [0, 1])
def test_restored_session_continues_bit_for_bit(form):
    from fusion_b200 import Session, mixed_config
    cfg = mixed_config(320, 240, 0.007)
    cfg.form = form
    p = synth.params(320, 240, synth.session_seed(4, 12), fx=cfg.fx, fy=cfg.fy, cx=cfg.cx, cy=cfg.cy,
                     depth_scale=5000.0)
    d, c, _ = synth.render(p, 0, 9)
    a = Session(cfg)
    for k in range(5):
        a.grab(d[k], c[k])
    snap = a.snapshot()
    rows_a = [_row(a.grab(d[k], c[k])) for k in range(5, 9)]
    b = Session(cfg)
    b.grab(d[0], c[0])                        # state to be overwritten
    b.restore(snap)
    rows_b = [_row(b.grab(d[k], c[k])) for k in range(5, 9)]
    assert rows_b == rows_a
    assert any(r[0] for r in rows_a)
    assert _digest(b) == _digest(a)
    a.close()
    b.close()


def test_snapshot_of_another_configuration_is_refused():
    from fusion_b200 import FusionError, Session, mixed_config
    a = Session(mixed_config(160, 120, 0.01))
    snap = a.snapshot()
    b = Session(mixed_config(160, 120, 0.012))
    with pytest.raises(FusionError):
        b.restore(snap)
    with pytest.raises(FusionError):
        a.restore(snap[:-1])
    a.close()
    b.close()
