"""Batched and served forms (fb_batch_*) through the C ABI.

Each session's result in a batch must be the one the same session gives
alone: the test runs ragged sessions (three resolutions, five voxel sizes,
independent seeded sequences) once alone through fb_grab_frame and once
together through fb_batch_step, in all three batch modes, with sessions
joining and skipping steps the way a server admits them -- so that steps of
more than three sessions (the group forms of the tracking kernels) and of
three (the forms of a session alone) alternate -- and compares every frame's
pose and counts and the final hash table and voxels bit for bit.  Mode 2
runs every stage kernel once for all sessions of a step (fused launches over
the concatenated grids); its sessions must still equal themselves alone, in
both map forms mixed in one step and with different raycast tiles.
"""
import hashlib

import numpy as np
import pytest

import rgbd_synth as synth
from fusion_b200.invariants import check_session

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")

SPECS = [(160, 120, 0.012, 11), (320, 240, 0.007, 12), (640, 480, 0.005, 13), (160, 120, 0.010, 14),
         (320, 240, 0.009, 15)]
N_FRAMES = 6


def _frames(w, h, seed, n):
    p = synth.params(w, h, synth.session_seed(4, seed), fx=525.0 * w / 640.0, fy=525.0 * w / 640.0,
                     cx=w / 2.0, cy=h / 2.0, depth_scale=5000.0)
    d, c, _ = synth.render(p, 0, n)
    return d, c


def _map_digest(sess):
    e = sess.entries()
    occ = e[:, 3] >= 0
    sdf, w, c = sess.blocks(e[occ][:, 3])
    h = hashlib.sha1()
    for a in (e, sdf.view(np.uint32), w, c):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest(), int(occ.sum())


def _row(r):
    return (r.tracked, r.tracker_state, r.fused, r.no_visible, r.no_allocated, r.no_new, r.error_flags,
            tuple(r.pose[:]), r.icp_count, r.rgb_count)


def _config(i, forms=None):
    from fusion_b200 import mixed_config
    w, h, v, _ = SPECS[i]
    c = mixed_config(w, h, v)
    if forms:
        c.form = forms[i]
    return c


def _alone(frames, schedule, forms=None):
    from fusion_b200 import Session
    out = []
    for i in range(len(SPECS)):
        s = Session(_config(i, forms))
        d, c = frames[i]
        rows = [_row(s.grab(d[k], c[k])) for k in range(len(schedule[i]))]
        out.append((rows, _map_digest(s)))
        assert check_session(s) == []
        s.close()
    return out


def _batched(frames, schedule, mode, tiles=None, forms=None, launch_stats=None, lanes=None):
    """schedule[i] = the steps at which session i has a frame."""
    from fusion_b200 import Batch, Session
    from fusion_b200.batch import set_raycast_tile
    sess = [Session(_config(i, forms)) for i in range(len(SPECS))]
    if tiles:
        for s, t in zip(sess, tiles):
            set_raycast_tile(s, *t)
    rows = [[] for _ in sess]
    nxt = [0] * len(sess)
    with Batch(mode=mode) as b:
        if lanes:
            b.set_lanes(lanes)
        n_steps = max(max(sch) for sch in schedule) + 1
        for step in range(n_steps):
            idx = [i for i in range(len(sess)) if step in schedule[i]]
            fr = []
            for i in idx:
                d, c = frames[i]
                fr.append((d[nxt[i]], c[nxt[i]]))
                nxt[i] += 1
            res = b.step([sess[i] for i in idx], fr)
            for i, r in zip(idx, res):
                rows[i].append(_row(r))
            if launch_stats is not None:
                launch_stats.append((len(idx), *b.launch_stats()))
        stats = b.stats()
    out = [(rows[i], _map_digest(s)) for i, s in enumerate(sess)]
    for s in sess:
        s.close()
    return out, stats


@pytest.fixture(scope="module")
def frames():
    return [_frames(w, h, seed, N_FRAMES) for (w, h, _, seed) in SPECS]


LOCKSTEP = [list(range(N_FRAMES))] * len(SPECS)
# session 1 joins at step 2, session 0 skips steps 3 and 4 (no frame arrived);
# steps of three sessions (steps 0 and 4: the tracking forms of sessions
# alone) alternate with steps of four (the group forms)
STAGGERED = [[0, 1, 2, 5, 6, 7], [2, 3, 4, 5, 6, 7], [0, 1, 2, 3, 4, 5], [0, 1, 3, 4, 6, 7],
             [1, 2, 3, 5, 6, 7]]


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("schedule", ["lockstep", "staggered"])
def test_each_session_in_the_batch_equals_it_alone(frames, mode, schedule):
    sch = LOCKSTEP if schedule == "lockstep" else STAGGERED
    alone = _alone(frames, sch)
    batched, (steps, captures) = _batched(frames, sch, mode)
    for i in range(len(SPECS)):
        assert batched[i][0] == alone[i][0], f"session {i}: per-frame results differ"
        assert batched[i][1] == alone[i][1], f"session {i}: final map differs"
    assert all(any(r[0] for r in rows) for rows, _ in alone)   # the sequences do track
    if mode == 1 and schedule == "lockstep":
        # compositions: init, then tracking without fusion for parities 0/1 ...
        assert captures <= steps


def test_raycast_tile_does_not_change_results(frames):
    base, _ = _batched(frames, LOCKSTEP, 0)
    tiled, _ = _batched(frames, LOCKSTEP, 0, tiles=[(0, 0), (32, 4), (8, 8)])
    assert tiled == base
    # fused steps: sessions with different tiles (and the queued raycast)
    # run as separate fused raycast launches
    fused, _ = _batched(frames, LOCKSTEP, 2, tiles=[(0, 0), (32, 4), (8, 8)])
    assert fused == base


def test_raycast_tile_change_between_frames_changes_no_result(frames):
    """The raycast dispatches its blocks in the order the z-range pass
    prepared from the last raycast's per-tile costs.  A session whose tile
    changes every frame (so each order comes from another tile grid's costs)
    gives the same poses, counts, map and final raycast maps as one that keeps
    the default tile."""
    from fusion_b200 import Session
    from fusion_b200.batch import set_raycast_tile
    d, c = frames[2]
    out = []
    for tiles in ([(16, 8)] * N_FRAMES, [(16, 8), (8, 8), (32, 4), (0, 0), (16, 8), (8, 16)]):
        s = Session(_config(2))
        rows = []
        for k in range(N_FRAMES):
            set_raycast_tile(s, *tiles[k])
            rows.append(_row(s.grab(d[k], c[k])))
        maps = [s.level(which, 0)[key].tobytes() for which in (0, 1) for key in ("vmap", "nmap")]
        out.append((rows, _map_digest(s), maps))
        s.close()
    assert out[0][0] == out[1][0]
    assert out[0][1] == out[1][1]
    assert out[0][2] == out[1][2]


FORMS = [1, 0, 1, 0, 0]   # precision and reference forms mixed in one step


@pytest.mark.parametrize("mode", [0, 2])
def test_two_batches_in_flight_equal_alone(frames, mode):
    """Two batches over disjoint sessions, each with one step in flight
    (fb_batch_submit / fb_batch_collect alternating), give every session its
    results alone."""
    from fusion_b200 import Batch, Session
    alone = _alone(frames, LOCKSTEP)
    sess = [Session(_config(i)) for i in range(len(SPECS))]
    halves = [[0, 2, 4], [1, 3]]
    rows = [[] for _ in sess]
    batches = [Batch(mode=mode), Batch(mode=mode)]
    for h, b in zip(halves, batches):
        b.submit([sess[i] for i in h], [(frames[i][0][0], frames[i][1][0]) for i in h])
    for k in range(N_FRAMES):
        for h, b in zip(halves, batches):
            res = b.collect()
            for i, r in zip(h, res):
                rows[i].append(_row(r))
            if k + 1 < N_FRAMES:
                b.submit([sess[i] for i in h], [(frames[i][0][k + 1], frames[i][1][k + 1]) for i in h])
    for b in batches:
        b.close()
    out = [(rows[i], _map_digest(s)) for i, s in enumerate(sess)]
    for s in sess:
        s.close()
    assert out == alone


def test_fused_step_mixes_map_forms(frames):
    """A fused step holding precision-form and reference-form sessions
    (different integration and raycast kernels, tracking sums compensated or
    not) gives every session its results alone."""
    alone = _alone(frames, STAGGERED, forms=FORMS)
    fused, _ = _batched(frames, STAGGERED, 2, forms=FORMS, lanes=2)
    for i in range(len(SPECS)):
        assert fused[i][0] == alone[i][0], f"session {i}: per-frame results differ"
        assert fused[i][1] == alone[i][1], f"session {i}: final map differs"


def test_fused_step_launch_count(frames):
    """A fused step makes about one frame's worth of launches whatever the
    number of sessions: each merged launch carries every session's kernel of
    that stage (a few more where sessions run different kernels -- two map
    forms, different tracker modes)."""
    stats = []
    one_lane, _ = _batched(frames, LOCKSTEP, 2, launch_stats=stats, lanes=1)
    alone = _alone(frames, LOCKSTEP)
    assert one_lane == alone
    print("(sessions, launches, per-session kernels) per step:", stats)
    for n, launches, kernels in stats:
        assert 0 < launches <= kernels
    # steady tracking steps: one frame's launches carry all five sessions'
    n, launches, kernels = stats[-1]
    assert n == len(SPECS)
    assert launches * (n - 1) < kernels, (launches, kernels)


def test_batch_rejects_a_session_twice(frames):
    from fusion_b200 import Batch, FusionError, Session, mixed_config
    s = Session(mixed_config(160, 120, 0.01))
    d, c = frames[0]
    with Batch() as b:
        with pytest.raises(FusionError):
            b.step([s, s], [(d[0], c[0]), (d[1], c[1])])
    s.close()


def test_recycled_frame_graphs_give_the_same_results():
    """A session whose frame graphs are rewritten from a closed session's
    executables (cudaGraphExecUpdate) gives the results of one whose graphs
    were instantiated.  A raycast tile no other test uses keeps these
    sessions' executables apart from the rest of the pool."""
    from fusion_b200 import Session, mixed_config
    from fusion_b200.batch import set_raycast_tile
    from fusion_b200.system import graph_exec_stats
    w, h, v, seed = SPECS[1]
    d, c = _frames(w, h, seed, N_FRAMES)
    d2, c2 = _frames(w, h, seed + 100, N_FRAMES)

    def run(voxel, dd, cc, close):
        s = Session(mixed_config(w, h, voxel))
        set_raycast_tile(s, 32, 2)
        rows = [_row(s.grab(dd[k], cc[k])) for k in range(N_FRAMES)]
        dig = _map_digest(s)
        if close:
            s.close()
        return s, rows, dig

    st0 = graph_exec_stats()
    a, rows_a, dig_a = run(v, d, c, close=False)
    st1 = graph_exec_stats()
    assert st1["instantiated"] > st0["instantiated"] and st1["updated"] == st0["updated"]
    run(0.011, d2, c2, close=True)      # its executables go back to the pool
    st2 = graph_exec_stats()
    _, rows_c, dig_c = run(v, d, c, close=True)
    st3 = graph_exec_stats()
    a.close()
    print("graph executables:", st0, st1, st2, st3)
    assert st3["updated"] > st2["updated"]
    assert st3["instantiated"] == st2["instantiated"]
    assert rows_c == rows_a
    assert dig_c == dig_a


def test_fused_step_of_more_sessions_than_one_launch_holds(frames):
    """A fused launch carries at most 32 sessions; a step of 34 sessions in
    one lane splits each stage into two launches, and every session still
    equals itself alone."""
    from fusion_b200 import Batch, Session, mixed_config
    w, h, v, _ = SPECS[0]
    d, c = frames[0]
    n, n_frames = 34, 3
    alone = []
    for _ in range(2):   # two sessions alone cover both halves of the check
        s = Session(mixed_config(w, h, v))
        alone.append([_row(s.grab(d[k], c[k])) for k in range(n_frames)])
        s.close()
    assert alone[0] == alone[1]
    sess = [Session(mixed_config(w, h, v)) for _ in range(n)]
    rows = [[] for _ in sess]
    with Batch(mode=2) as b:
        b.set_lanes(1)
        for k in range(n_frames):
            for i, r in enumerate(b.step(sess, [(d[k], c[k])] * n)):
                rows[i].append(_row(r))
            launches, kernels = b.launch_stats()
            assert launches < kernels
    for s in sess:
        s.close()
    assert all(r == alone[0] for r in rows)


def test_batch_call_errors(frames):
    from fusion_b200 import Batch, FusionError, Session, mixed_config
    w, h, v, _ = SPECS[0]
    d, c = frames[0]
    s = Session(mixed_config(w, h, v))
    with Batch() as b:
        with pytest.raises(FusionError):
            b.set_mode(3)
        with pytest.raises(FusionError):
            b.set_lanes(0)
        with pytest.raises(FusionError):
            b.set_lanes(33)
        with pytest.raises(FusionError):
            b._pending = (1, None, None, None)
            b.collect()                        # nothing submitted
        b.submit([s], [(d[0], c[0])])
        with pytest.raises(FusionError):
            b.submit([s], [(d[1], c[1])])      # one step in flight per batch
        r = b.collect()
        assert len(r) == 1 and r[0].tracked
    s.close()


def test_integration_grid_does_not_change_results(frames):
    from fusion_b200.batch import set_integration_grid
    base, _ = _batched(frames, LOCKSTEP, 0)
    from fusion_b200 import Batch, Session
    sess = [Session(_config(i)) for i in range(len(SPECS))]
    for s, g in zip(sess, [1, 2, 16, 0, 4]):
        set_integration_grid(s, g)
    rows = [[] for _ in sess]
    with Batch(mode=2) as b:
        for k in range(N_FRAMES):
            res = b.step(sess, [(frames[i][0][k], frames[i][1][k]) for i in range(len(sess))])
            for i, r in enumerate(res):
                rows[i].append(_row(r))
    out = [(rows[i], _map_digest(s)) for i, s in enumerate(sess)]
    for s in sess:
        s.close()
    assert out == base
