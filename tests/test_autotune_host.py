"""The batched form's autotuner (fusion_b200/batch.py) on the host with a
fake batch whose step time depends on each group's tile, integration grid
and the lanes: every group gets its fastest candidate, groups are tuned one
after another with the others left as they are, and every timed step is a
real step of the workload (no GPU)."""
import time

from fusion_b200 import batch as B


class FakeCfg:
    def __init__(self, w, h, v=0.01):
        self.width, self.height, self.voxel_size = w, h, v


class FakeSession:
    def __init__(self, w, h, v=0.01):
        self.cfg = FakeCfg(w, h, v)
        self.tile = (16, 8)
        self.grid = 0


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


GRID_BEST = {(320, 240, 0): 4, (320, 240, 2): 16, (640, 480, 1): 2}


class GridBatch:
    def __init__(self):
        self.steps = 0
        self.mode = 2
        self.lanes = 4

    def set_lanes(self, lanes):
        self.lanes = lanes

    def step(self, sessions, frames, on_device=False):
        self.steps += 1
        slow = {(s.cfg.width, s.cfg.height, B.voxel_bucket(s.cfg.voxel_size)) for s in sessions
                if s.grid != GRID_BEST[(s.cfg.width, s.cfg.height, B.voxel_bucket(s.cfg.voxel_size))]}
        time.sleep(0.003 * len(slow) + (0.003 if self.lanes != 2 else 0.0))


def test_integration_grids_and_lanes(monkeypatch):
    monkeypatch.setattr(B, "set_integration_grid", lambda s, g: setattr(s, "grid", g))
    sessions = [FakeSession(320, 240, 0.005), FakeSession(320, 240, 0.018), FakeSession(640, 480, 0.01),
                FakeSession(320, 240, 0.006)]
    fb = GridBatch()
    chosen, taken = B.autotune_integration_grids(fb, sessions, lambda: [None] * len(sessions), steps_per=2)
    assert chosen == GRID_BEST
    assert all(s.grid == GRID_BEST[(s.cfg.width, s.cfg.height, B.voxel_bucket(s.cfg.voxel_size))]
               for s in sessions)
    assert taken == fb.steps == 3 * len(B.GRID_CANDIDATES) * 3
    lanes, taken2 = B.autotune_lanes(fb, sessions, lambda: [None] * len(sessions), steps_per=2)
    assert lanes == 2 and fb.lanes == 2
    assert taken2 == 4 * len(B.LANE_CANDIDATES)
