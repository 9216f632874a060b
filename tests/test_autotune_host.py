"""The raycast-tile autotuner (fusion_b200/batch.py) on the host with a fake
batch whose step time depends on each resolution group's tile: every group
gets its fastest candidate, groups are tuned one after another with the
others left as they are, and every timed step is a real step of the
workload (no GPU)."""
import time

from fusion_b200 import batch as B


class FakeCfg:
    def __init__(self, w, h):
        self.width, self.height = w, h


class FakeSession:
    def __init__(self, w, h):
        self.cfg = FakeCfg(w, h)
        self.tile = (16, 8)


BEST = {(320, 240): (8, 8), (640, 480): (32, 4)}


class FakeBatch:
    def __init__(self):
        self.steps = 0

    def step(self, sessions, frames, on_device=False):
        assert len(frames) == len(sessions)
        self.steps += 1
        # 3 ms for every group whose tile is not its best
        slow = {(s.cfg.width, s.cfg.height) for s in sessions if s.tile != BEST[(s.cfg.width, s.cfg.height)]}
        time.sleep(0.003 * len(slow))


def test_each_group_gets_its_fastest_tile(monkeypatch):
    monkeypatch.setattr(B, "set_raycast_tile", lambda s, bx, by: setattr(s, "tile", (bx, by)))
    sessions = [FakeSession(320, 240), FakeSession(640, 480), FakeSession(320, 240), FakeSession(640, 480)]
    fb = FakeBatch()
    frames_served = []

    def next_frames():
        frames_served.append(1)
        return [None] * len(sessions)

    cands = [(16, 8), (8, 8), (32, 4)]
    chosen, taken = B.autotune_raycast_tiles(fb, sessions, next_frames, candidates=cands, steps_per=2)
    assert chosen == BEST
    assert all(s.tile == BEST[(s.cfg.width, s.cfg.height)] for s in sessions)
    assert taken == fb.steps == len(frames_served) == 2 * len(cands) * 3
