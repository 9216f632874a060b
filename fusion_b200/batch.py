"""Batched and served forms: many independent sessions on one GPU.

`Batch` steps a set of sessions -- any resolutions, cameras and voxel sizes --
by one frame each through fb_batch_step, with all of their frames in flight on
the device together.  Each session's result is exactly what `Session.grab`
gives for the same input on that session alone: the same kernel bodies run on
the same data -- in per-session launches, or in fused launches that carry
every session's part (mode 2) -- only concurrently.

`mixed_population` draws the ragged session mix of the batched and served
configurations (resolution from {160x120, 320x240, 640x480}, voxel size
uniform in 4-20 mm) and `mixed_config` sizes each session's map for its voxel
size.  `autotune_batch` picks, by timing real steps of the batch, each
resolution's raycast tile (the CUDA block shape of the model raycast), each
(resolution, voxel-size class)'s integration grid and, for fused steps, the
number of lanes -- shapes that change no result.
"""
import ctypes
import math
import time

import numpy as np

from . import _lib
from ._lib import FrameInput, FrameResult, check
from .system import make_config

RESOLUTIONS = ((160, 120), (320, 240), (640, 480))
TILE_CANDIDATES = ((0, 0), (16, 8), (8, 8), (32, 4), (8, 16), (16, 4), (32, 2))


def _next_pow2(v):
    return 1 << max(0, int(math.ceil(math.log2(max(1, v)))))


def mixed_config(width, height, voxel_size, trunc_voxels=4):
    """Session configuration for a width x height camera with `voxel_size`
    metre voxels: pool sized for a 4 x 4 x 3 m room seen from all sides
    (160 000 blocks at 5 mm, scaling with the surface area in blocks, i.e.
    1 / voxel_size^2), rounded up to a power of two in [2^13, 2^19]; buckets =
    4 x blocks and excess = blocks (the full-size configuration's ratios)."""
    blocks = _next_pow2(int(math.ceil(160000 * (0.005 / voxel_size) ** 2)))
    blocks = min(max(blocks, 1 << 13), 1 << 19)
    return make_config(width, height, voxel_size, trunc_voxels, 4 * blocks, blocks, blocks)


def mixed_population(n, seed):
    """n (width, height, voxel_size) triples: resolution uniform over
    RESOLUTIONS, voxel size uniform in [4, 20] mm (float32-rounded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
        v = float(np.float32(rng.uniform(0.004, 0.020)))
        out.append((w, h, v))
    return out


class Batch:
    """fb_batch: mode 0 launches each session's frame graph on its own stream;
    mode 1 captures one graph per composition of the step; mode 2 (fused)
    runs each stage kernel once for all sessions of the step."""

    def __init__(self, mode=0, stream=None):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        check("fb_batch_create", self.lib.fb_batch_create(stream, ctypes.byref(h)))
        self.h = h
        self.set_mode(mode)

    def set_mode(self, mode):
        check("fb_batch_set_mode", self.lib.fb_batch_set_mode(self.h, int(mode)))
        self.mode = int(mode)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _inputs(self, sessions, frames, on_device):
        n = len(sessions)
        hs = (ctypes.c_void_p * n)(*[s.h.value for s in sessions])
        ins = (FrameInput * n)()
        keep = []
        for i, (s, (d, c)) in enumerate(zip(sessions, frames)):
            W = s.cfg.width
            if on_device:
                ins[i] = FrameInput(d.data_ptr(), 2 * W, c.data_ptr(), 3 * W, 1)
            else:
                d = np.ascontiguousarray(d, np.uint16)
                c = np.ascontiguousarray(c, np.uint8)
                keep.append((d, c))
                ins[i] = FrameInput(d.ctypes.data, d.strides[0], c.ctypes.data, c.strides[0], 0)
        return hs, ins, keep

    def step(self, sessions, frames, on_device=False):
        """One frame per session.  frames[i] = (depth u16 [H, W], rgb u8
        [H, W, 3]): numpy arrays, or with on_device objects with data_ptr()
        (contiguous device memory).  Returns one FrameResult per session."""
        n = len(sessions)
        hs, ins, keep = self._inputs(sessions, frames, on_device)
        out = (FrameResult * n)()
        check("fb_batch_step", self.lib.fb_batch_step(self.h, hs, n, ins, out))
        return list(out)

    def submit(self, sessions, frames, on_device=False):
        """The first half of step(): starts the step and returns at once.
        The frames (kept alive here) are read until collect()."""
        hs, ins, keep = self._inputs(sessions, frames, on_device)
        check("fb_batch_submit", self.lib.fb_batch_submit(self.h, hs, len(sessions), ins))
        self._pending = (len(sessions), hs, ins, keep)

    def collect(self):
        """Waits for the submitted step; one FrameResult per session."""
        n = self._pending[0]
        out = (FrameResult * n)()
        check("fb_batch_collect", self.lib.fb_batch_collect(self.h, out))
        self._pending = None
        return list(out)

    def reserve(self, nbytes):
        """Map `nbytes` of device memory into the pool sessions allocate from."""
        check("fb_batch_reserve", self.lib.fb_batch_reserve(self.h, int(nbytes)))

    def stats(self):
        steps, caps = ctypes.c_uint64(), ctypes.c_uint64()
        check("fb_batch_stats", self.lib.fb_batch_stats(self.h, ctypes.byref(steps), ctypes.byref(caps)))
        return steps.value, caps.value

    def set_lanes(self, lanes):
        """Mode 2: number of session groups whose fused launches overlap."""
        check("fb_batch_set_lanes", self.lib.fb_batch_set_lanes(self.h, int(lanes)))

    def launch_stats(self):
        """Mode 2: (kernel launches of the last step, per-session kernels they carried)."""
        launches, kernels = ctypes.c_int(), ctypes.c_int()
        check("fb_batch_launch_stats",
              self.lib.fb_batch_launch_stats(self.h, ctypes.byref(launches), ctypes.byref(kernels)))
        return launches.value, kernels.value


def set_raycast_tile(session, bx, by):
    check("fb_session_set_raycast_tile", session.lib.fb_session_set_raycast_tile(session.h, bx, by))


def set_integration_grid(session, ctas_per_sm):
    check("fb_session_set_integration_grid",
          session.lib.fb_session_set_integration_grid(session.h, int(ctas_per_sm)))


def voxel_bucket(voxel_size):
    """Coarse voxel-size class of a session for the integration autotuner:
    the visible-block count, and so the integration's work, scales with
    1 / voxel_size^2."""
    return 0 if voxel_size < 0.008 else 1 if voxel_size < 0.014 else 2


def _tune_groups(batch, sessions, next_frames, key, candidates, apply, steps_per, on_device):
    """For each group of sessions (by key(session)), one after another with
    the other groups left as they are: every candidate applied to the whole
    group, one step that rebuilds the frame graphs, `steps_per` timed steps
    of the real workload; the fastest candidate is kept.  Returns
    {group: candidate} and the number of steps taken."""
    groups = {}
    for s in sessions:
        groups.setdefault(key(s), []).append(s)
    chosen, taken = {}, 0
    for g, members in sorted(groups.items()):
        best, best_t = None, float("inf")
        for cand in candidates:
            for s in members:
                apply(s, cand)
            batch.step(sessions, next_frames(), on_device=on_device)   # graphs rebuilt here
            taken += 1
            t0 = time.perf_counter()
            for _ in range(steps_per):
                batch.step(sessions, next_frames(), on_device=on_device)
            t = (time.perf_counter() - t0) / steps_per
            taken += steps_per
            if t < best_t:
                best, best_t = cand, t
        for s in members:
            apply(s, best)
        chosen[g] = best
    return chosen, taken


def autotune_raycast_tiles(batch, sessions, next_frames, candidates=TILE_CANDIDATES, steps_per=2,
                           on_device=False):
    """Pick the raycast tile of every resolution group of `sessions` by
    timing batch steps: groups one after another, each candidate applied to
    the whole group for `steps_per` steps (after one step that rebuilds the
    frame graphs), the fastest kept.  next_frames() returns the next frame of
    every session (the steps are real frames of the workload).  Returns
    {(width, height): (bx, by)} and the number of steps taken."""
    return _tune_groups(batch, sessions, next_frames, lambda s: (s.cfg.width, s.cfg.height), candidates,
                        lambda s, t: set_raycast_tile(s, *t), steps_per, on_device)


GRID_CANDIDATES = (0, 2, 4, 16)


def autotune_integration_grids(batch, sessions, next_frames, candidates=GRID_CANDIDATES, steps_per=2,
                               on_device=False):
    """Pick the integration grid (CTAs per SM, 0 = the form's default) of
    every (resolution, voxel-size class) group the same way.  Returns
    {(width, height, class): ctas_per_sm} and the number of steps taken."""
    return _tune_groups(batch, sessions, next_frames,
                        lambda s: (s.cfg.width, s.cfg.height, voxel_bucket(s.cfg.voxel_size)), candidates,
                        set_integration_grid, steps_per, on_device)


LANE_CANDIDATES = (1, 2, 4, 8)


def autotune_lanes(batch, sessions, next_frames, candidates=LANE_CANDIDATES, steps_per=2, on_device=False):
    """Fused steps (batch mode 2): the number of lanes, timed the same way
    (one step to build the new plans and graphs, then `steps_per` steps).
    Returns (lanes, steps taken)."""
    best, best_t, taken = None, float("inf"), 0
    for lanes in candidates:
        batch.set_lanes(lanes)
        for _ in range(2):   # a composition runs as a graph from its second use
            batch.step(sessions, next_frames(), on_device=on_device)
        taken += 2
        t0 = time.perf_counter()
        for _ in range(steps_per):
            batch.step(sessions, next_frames(), on_device=on_device)
        t = (time.perf_counter() - t0) / steps_per
        taken += steps_per
        if t < best_t:
            best, best_t = lanes, t
    batch.set_lanes(best)
    return best, taken


def autotune_batch(batch, sessions, next_frames, steps_per=2, on_device=False):
    """The batched form's block and tile shapes, picked on the real workload:
    the raycast tile per resolution, the integration grid per resolution and
    voxel-size class, and (fused steps) the number of lanes.  Results do not
    depend on any of them.  Returns {"raycast_tiles", "integration_grids",
    "lanes", "steps"}."""
    tiles, n1 = autotune_raycast_tiles(batch, sessions, next_frames, steps_per=steps_per, on_device=on_device)
    grids, n2 = autotune_integration_grids(batch, sessions, next_frames, steps_per=steps_per, on_device=on_device)
    lanes, n3 = None, 0
    if getattr(batch, "mode", 0) == 2:
        lanes, n3 = autotune_lanes(batch, sessions, next_frames, steps_per=steps_per, on_device=on_device)
    return {"raycast_tiles": tiles, "integration_grids": grids, "lanes": lanes, "steps": n1 + n2 + n3}
