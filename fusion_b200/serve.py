"""Served form: a request loop fusing frames of many independent sessions as
they arrive, on one GPU.

Clients (camera sessions) arrive over time, stream frames as a Poisson
process (30 Hz by default) for a lognormal lifetime, and leave.  A client is
admitted when its session's device memory (fb_session_bytes) fits in the HBM
budget beside the sessions already resident, else it waits in a FIFO queue
until departures free enough memory.  Each admitted client's hash table,
voxel blocks, frames and pose stay on the device for its whole life.

The loop is continuous batching: whenever frames are pending, every client
with a pending frame contributes its oldest one to the next fb_batch_step
(at most `max_batch` clients, oldest frame first); frames that arrive while a
step is on the GPU go into the following step.  A frame's latency runs from
its arrival time to the end of the step that fused it.  Each client's results
are the ones its session would give alone (fb_batch_step's guarantee), so
batching changes latency and throughput only.

Frames come from a pool of pre-rendered seeded sequences per resolution
(pinned host memory; a client plays its sequence forwards then backwards so
that the camera motion stays continuous), copied to the device inside each
step.
"""
import heapq
import math
import time

import numpy as np

import rgbd_synth as synth

from . import _lib
from .batch import RESOLUTIONS, Batch, mixed_config


def sequence_seeds(config_id, count, width=160, height=120, max_median_depth=2.0, limit=1000):
    """The first `count` session indices of `config_id` whose first frame's
    median valid depth is at most `max_median_depth` metres.  Beyond ~2 m the
    generator's depth noise (0.0012 + 0.0019 (z - 0.4)^2 m) approaches the
    truncation band of the small-voxel sessions and the reference's tracker
    loses such sequences at their first frame (the FP64 oracle agrees), which
    would leave them untracked -- doing no fusion or raycast -- for the rest of
    their life."""
    out = []
    for i in range(limit):
        seed = synth.session_seed(config_id, i)
        p = synth.params(width, height, seed, fx=525.0 * width / 640.0, fy=525.0 * width / 640.0,
                         cx=width / 2.0, cy=height / 2.0, depth_scale=5000.0)
        d, _, _ = synth.render(p, 0, 1)
        v = d[0][d[0] > 0]
        if v.size and np.median(v) / 5000.0 <= max_median_depth:
            out.append(seed)
            if len(out) == count:
                break
    return out


class FramePool:
    """Pre-rendered sequences per resolution, pinned host memory."""

    def __init__(self, seeds, n_frames, resolutions=RESOLUTIONS, pin=True):
        import torch
        self.seq = {}
        for (w, h) in resolutions:
            for k, seed in enumerate(seeds):
                p = synth.params(w, h, seed, fx=525.0 * w / 640.0, fy=525.0 * w / 640.0, cx=w / 2.0,
                                 cy=h / 2.0, depth_scale=5000.0)
                d, c, _ = synth.render(p, 0, n_frames)
                if pin:
                    d = torch.from_numpy(d).pin_memory().numpy()
                    c = torch.from_numpy(c).pin_memory().numpy()
                self.seq[(w, h, k)] = (d, c)
        self.n_seq = len(seeds)
        self.n_frames = n_frames

    def frame(self, w, h, k, i):
        """Frame i of sequence k played forwards then backwards."""
        n = self.n_frames
        period = 2 * n - 2 if n > 1 else 1
        j = i % period
        if j >= n:
            j = period - j
        d, c = self.seq[(w, h, k)]
        return d[j], c[j]


class Client:
    def __init__(self, cid, width, height, voxel, seq, t_arrive, lifetime, rate, rng):
        self.cid, self.width, self.height, self.voxel, self.seq = cid, width, height, voxel, seq
        self.t_arrive, self.lifetime, self.rate = t_arrive, lifetime, rate
        self.rng = rng
        self.session = None
        self.t_admit = None
        self.t_end = None
        self.pending = []       # arrival times of frames not yet fused
        self.next_arrival = None
        self.sent = 0           # frames taken from the sequence so far
        self.bytes = 0
        self.load = 0.0         # GPU milliseconds per second while admitted


def make_clients(n, seed, rate=30.0, median_life=20.0, life_sigma=0.5, horizon=0.0):
    """n clients present at t = 0 (the steady-state population) plus clients
    arriving as a Poisson process at n / (mean lifetime) per second over
    `horizon` seconds, which keeps the population steady.  Lifetimes are
    lognormal (median `median_life` s), frame rate `rate` Hz, resolution
    uniform over RESOLUTIONS, voxel size uniform in [4, 20] mm."""
    rng = np.random.default_rng(seed)
    mean_life = median_life * math.exp(life_sigma ** 2 / 2)
    times = [0.0] * n
    t = rng.exponential(mean_life / n)
    while t < horizon:
        times.append(t)
        t += rng.exponential(mean_life / n)
    out = []
    for i, ta in enumerate(times):
        w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
        v = float(np.float32(rng.uniform(0.004, 0.020)))
        life = float(rng.lognormal(math.log(median_life), life_sigma))
        out.append(Client(i, w, h, v, 0, ta, life, rate, np.random.default_rng(seed * 1000003 + i)))
    return out


class Admission:
    """Admission control.  A client is admitted when its session's device
    memory (`need(c)` bytes) fits in the HBM budget beside the resident
    sessions and -- when per-frame GPU costs are known -- when its expected
    GPU time per second of wall time (frame rate x the per-frame cost of its
    resolution) fits beside theirs under `load_max` of the GPU.  The compute
    test keeps the admitted load below saturation, so that admitted clients
    keep their latency when more clients arrive than one GPU can serve; the
    rest wait in FIFO order (head-of-line: a later, smaller client does not
    pass the head).  The costs come from batch steps of a few sessions
    (Server.calibrate); larger batches overlap more of each frame's
    latency-bound work, so the GPU saturates above a load of 1.0 by that
    measure: on B200 at about 1.25 for the mixed-resolution population
    (p99 18 ms at 1.2, 54 ms at 1.3), hence the default of 1.15."""

    def __init__(self, budget_bytes, need, frame_cost_ms=None, load_max=1.15):
        self.budget = float(budget_bytes)
        self.need = need
        self.cost = dict(frame_cost_ms) if frame_cost_ms else None
        self.load_max = float(load_max)
        self.reserved = 0.0
        self.load = 0.0          # admitted GPU milliseconds per second
        self.peak = 0.0
        self.peak_load = 0.0

    def gpu_ms_per_s(self, c):
        return c.rate * self.cost[(c.width, c.height)] if self.cost else 0.0

    def fits(self, c):
        if self.reserved + self.need(c) > self.budget:
            return False
        return self.cost is None or self.load + self.gpu_ms_per_s(c) <= self.load_max * 1000.0

    def take(self, c):
        c.bytes = self.need(c)
        c.load = self.gpu_ms_per_s(c)
        self.reserved += c.bytes
        self.load += c.load
        self.peak = max(self.peak, self.reserved)
        self.peak_load = max(self.peak_load, self.load)

    def release(self, c):
        self.reserved -= c.bytes
        self.load -= c.load


class Server:
    """The request loop.  Admission work -- creating a session (one
    stream-ordered allocation from memory reserved up front, map reset) and
    capturing its frame graphs -- is done by the step loop itself in slices
    between steps: at most one session creation or one graph capture per
    iteration, so that no step waits for more than one slice (graph
    instantiation holds driver locks that a second host thread's launches
    and copies would wait for, which showed as 100+ ms stalls).  A session
    captures two sets of frame graphs: those of batch steps with other
    sessions, then those of steps of one to three sessions (the library picks
    the set by the step's size; both give the same results).  A client
    becomes active, and its frames start arriving, once its session is ready.
    Clients present at the start are admitted before the clock starts.
    Admission (class Admission) is by the HBM budget and, once calibrate()
    has measured the per-resolution frame costs, by GPU load.

    pipeline: how many batch steps may be in flight at once (fb_batch_submit
    / fb_batch_collect on that many batches).  With two, the loop submits
    the ready clients' frames while another step runs, and collects the
    oldest step when no further step can start (every batch busy, or every
    ready client already in flight): one step's last kernels overlap the
    next one's first.  A client has at most one frame in flight."""

    def __init__(self, pool, budget_bytes=120e9, mode=0, max_batch=256, frame_cost_ms=None, load_max=1.15,
                 pipeline=1):
        import torch
        self.lib = _lib.load()
        self.pool = pool
        self.budget = float(budget_bytes)
        self.batch = Batch(mode=mode)
        self.batches = [self.batch] + [Batch(mode=mode) for _ in range(max(1, int(pipeline)) - 1)]
        self.max_batch = max_batch
        self.frame_cost_ms = dict(frame_cost_ms) if frame_cost_ms else None
        self.load_max = float(load_max)
        # one stream for every session's own work (creation, graph capture):
        # creating a stream per session while frames run can stall the loop
        # for tens of milliseconds
        self._stream = torch.cuda.Stream()
        self.stream = self._stream.cuda_stream

    def close(self):
        for b in self.batches:
            b.close()

    def _need(self, c):
        return float(self.lib.fb_session_bytes(mixed_config(c.width, c.height, c.voxel)))

    def calibrate(self, resolutions=RESOLUTIONS, sessions=8, voxel=0.012, steps=6, warmup=3):
        """Per-frame GPU cost of each resolution, for compute admission: the
        wall time of batch steps of `sessions` sessions of that resolution
        (frames copied from the pool's pinned host memory, as in serving)
        divided by the frames fused.  Sets and returns {(w, h): ms}."""
        from .system import Session
        cost = {}
        for (w, h) in resolutions:
            group = [Session(mixed_config(w, h, voxel), stream=self.stream) for _ in range(sessions)]
            for g in group:
                g.prepare(shared=True)
            for i in range(warmup + steps):
                if i == warmup:
                    t = time.perf_counter()
                frames = [self.pool.frame(w, h, k % self.pool.n_seq, i) for k in range(sessions)]
                self.batch.step(group, frames)
            cost[(w, h)] = (time.perf_counter() - t) * 1e3 / (steps * sessions)
            for g in group:
                g.close()
        self.frame_cost_ms = cost
        return cost

    def run(self, clients, duration):
        """Serve `clients` for `duration` seconds of wall time.  Returns the
        statistics of the run."""
        from .system import Session, graph_exec_stats
        for k, c in enumerate(clients):
            c.seq = k % self.pool.n_seq
        by_id = {c.cid: c for c in clients}
        waiting, active, preparing, to_open = [], {}, [], []
        adm = Admission(self.budget, self._need, self.frame_cost_ms, self.load_max)
        lat, batch_sizes, wait_times = [], [], []
        worst = {"step_ms": 0.0, "step_with_new_session_ms": 0.0, "create_ms": 0.0, "capture_ms": 0.0,
                 "close_ms": 0.0}
        admitted = queued = 0
        events = []      # (time, kind 0 arrive / 1 leave, id)

        # device memory for the sessions expected at once (those present at the
        # start and as many again for arrivals, within the budget), mapped
        # before the clock starts
        warm_bytes = sum(self._need(c) for c in clients if c.t_arrive <= 0)
        self.batch.reserve(min(self.budget, 2.0 * warm_bytes))
        warm = []
        for c in clients:
            if c.t_arrive > 0:
                heapq.heappush(events, (c.t_arrive, 0, c.cid))
                continue
            if not waiting and adm.fits(c):
                adm.take(c)
                c.session = Session(mixed_config(c.width, c.height, c.voxel), stream=self.stream)
                c.session.prepare(shared=True)
                c.session.prepare(shared=False)
                warm.append(c)
            else:
                waiting.append(c)
                queued += 1
        # frame-graph executables for the sessions expected to arrive, made
        # before the clock and released into the library's executable pool:
        # an arriving session's capture then rewrites one of them
        # (cudaGraphExecUpdate) instead of instantiating a graph while other
        # sessions' frames run, which stalled the loop for up to 80 ms
        # (held open together, as far as the budget allows, so that each
        # arrival finds its own set of executables)
        group, held = [], adm.reserved
        for c in clients:
            if c.t_arrive <= 0 and c.session is not None:
                continue
            need = self._need(c)
            if group and held + need > self.budget:
                for g in group:
                    g.close()
                group, held = [], adm.reserved
            g = Session(mixed_config(c.width, c.height, c.voxel), stream=self.stream)
            g.prepare(shared=True)
            g.prepare(shared=False)
            group.append(g)
            held += need
        for g in group:
            g.close()
        ex0 = graph_exec_stats()
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        def activate(c, t):
            nonlocal admitted
            c.t_admit = t
            c.t_end = t + c.lifetime
            c.next_arrival = t + c.rng.exponential(1.0 / c.rate)
            active[c.cid] = c
            heapq.heappush(events, (c.t_end, 1, c.cid))
            admitted += 1
            if c.t_admit > c.t_arrive + 1e-6:
                wait_times.append(c.t_admit - c.t_arrive)

        def reserve_for(c):
            adm.take(c)
            to_open.append(c)

        def admit_waiting():
            while waiting and adm.fits(waiting[0]):
                reserve_for(waiting.pop(0))

        def admission_slice():
            """One session creation or one graph capture."""
            t_s = time.perf_counter()
            if preparing:
                # the graphs of steps with other sessions, then those of
                # steps alone (batch steps of one to three sessions)
                c = preparing[0]
                if c.session.prepare_some(0, shared=True) > 0:
                    c.session.prepare_some(1, shared=True)
                elif c.session.prepare_some(1, shared=False) == 0:
                    preparing.pop(0)
                    activate(c, now())
                key = "capture_ms"
            elif to_open:
                c = to_open.pop(0)
                c.session = Session(mixed_config(c.width, c.height, c.voxel), stream=self.stream)
                preparing.append(c)
                key = "create_ms"
            else:
                return
            worst[key] = max(worst[key], (time.perf_counter() - t_s) * 1e3)

        free = list(range(len(self.batches)))
        inflight = []    # (batch, clients, frames, submit time), oldest first
        for c in clients:
            c.in_flight = c.leaving = False

        def close_client(c):
            t_c = time.perf_counter()
            c.session.close()
            worst["close_ms"] = max(worst["close_ms"], (time.perf_counter() - t_c) * 1e3)
            c.session = None
            adm.release(c)
            admit_waiting()

        def collect_oldest():
            b, ready, _, t_s = inflight.pop(0)
            self.batches[b].collect()
            t_done = now()
            key = "step_with_new_session_ms" if any(c.sent < 2 for c in ready) else "step_ms"
            worst[key] = max(worst[key], (t_done - t_s) * 1e3)
            for c in ready:
                lat.append(t_done - c.pending.pop(0))
                c.sent += 1
                c.in_flight = False
                if c.leaving:
                    c.leaving = False
                    close_client(c)
            batch_sizes.append(len(ready))
            free.append(b)

        for c in warm:
            activate(c, 0.0)
        try:
            while True:
                t = now()
                if t >= duration:
                    break
                while events and events[0][0] <= t:
                    _, kind, cid = heapq.heappop(events)
                    c = by_id[cid]
                    if kind == 0:
                        if not waiting and adm.fits(c):
                            reserve_for(c)
                        else:
                            waiting.append(c)
                            queued += 1
                    elif cid in active:
                        del active[cid]
                        if c.in_flight:
                            c.leaving = True    # closed when its step is collected
                        else:
                            close_client(c)
                if preparing or to_open:
                    admission_slice()
                for c in active.values():
                    while c.next_arrival is not None and c.next_arrival <= t and c.next_arrival < c.t_end:
                        c.pending.append(c.next_arrival)
                        c.next_arrival += c.rng.exponential(1.0 / c.rate)
                ready = sorted((c for c in active.values() if c.pending and not c.in_flight),
                               key=lambda c: c.pending[0])
                if ready and free:
                    ready = ready[:self.max_batch]
                    frames = [self.pool.frame(c.width, c.height, c.seq, c.sent) for c in ready]
                    b = free.pop(0)
                    t_s = now()
                    self.batches[b].submit([c.session for c in ready], frames)
                    for c in ready:
                        c.in_flight = True
                    inflight.append((b, ready, frames, t_s))
                    continue
                if inflight:
                    collect_oldest()
                    continue
                if not (preparing or to_open):
                    nxt = min([c.next_arrival for c in active.values() if c.next_arrival is not None] +
                              ([events[0][0]] if events else []) + [duration])
                    time.sleep(max(0.0, min(nxt - now(), 0.001)))
            while inflight:
                collect_oldest()
            wall = now()
        finally:
            # no session is closed while a step holding it may still run
            for b, _, _, _ in inflight:
                try:
                    self.batches[b].collect()
                except Exception:
                    pass
            for c in clients:
                if c.session is not None:
                    c.session.close()
                    c.session = None
        lat_ms = np.array(lat) * 1e3 if lat else np.zeros(1)
        backlog = sum(len(c.pending) for c in clients)
        ex1 = graph_exec_stats()
        return {
            "frames": len(lat), "wall_s": wall, "frames_per_s": len(lat) / wall,
            "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                           "max": float(lat_ms.max())},
            "steps": len(batch_sizes), "mean_batch": float(np.mean(batch_sizes)) if batch_sizes else 0.0,
            "clients": len(clients), "admitted": admitted, "queued": queued,
            "still_queued_at_end": len(waiting),
            "mean_wait_s": float(np.mean(wait_times)) if wait_times else 0.0,
            "backlog_frames_at_end": backlog, "peak_reserved_bytes": adm.peak, "budget_bytes": self.budget,
            "admission": ({"frame_cost_ms": {f"{w}x{h}": v for (w, h), v in adm.cost.items()},
                           "load_max": adm.load_max, "peak_admitted_load": adm.peak_load / 1000.0}
                          if adm.cost else "memory only"),
            "worst_host_ms": worst,
            "graph_captures": {"updated": ex1["updated"] - ex0["updated"],
                               "instantiated": ex1["instantiated"] - ex0["instantiated"]},
        }
