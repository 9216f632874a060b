"""The served form's request loop (fusion_b200/serve.py) on the host with
fakes for the sessions, the batch and the frame pool (no GPU): arrivals are
admitted in order, each session captures both sets of frame graphs (steps
of other sessions, then steps alone) one capture per admission slice before
its first frame, frames are stepped in batches of the clients with pending
frames, and departures close sessions -- with two steps in flight too,
where no session is closed, and no client stepped, while its step runs."""
import time

from fusion_b200 import serve
from fusion_b200 import system as S

GRAPHS = 10   # frame graphs per set (tracker modes x fusion x parity)


class FakeSession:
    made = []

    def __init__(self, cfg, stream=None):
        self.missing = {True: GRAPHS, False: GRAPHS}
        self.calls = []           # (max_graphs, shared) of every prepare_some
        self.closed = False
        self.steps = 0
        FakeSession.made.append(self)

    def prepare(self, shared=False):
        self.missing[shared] = 0

    def prepare_some(self, max_graphs=1, shared=False):
        self.calls.append((max_graphs, shared))
        self.missing[shared] = max(0, self.missing[shared] - max_graphs)
        return self.missing[shared]

    def close(self):
        assert not getattr(self, "in_flight", False), "session closed while its step runs"
        self.closed = True


class FakeBatch:
    def __init__(self):
        self.sizes = []
        self.unready = 0
        self.pending = None
        self.overlapped = 0

    def reserve(self, n):
        pass

    def step(self, sessions, frames):
        self.submit(sessions, frames)
        time.sleep(0.001)
        self.collect()

    def submit(self, sessions, frames):
        assert self.pending is None
        self.sizes.append(len(sessions))
        for s in sessions:
            assert not getattr(s, "in_flight", False), "a session in two steps at once"
            s.in_flight = True
            s.steps += 1
            if s.missing[True] or s.missing[False]:
                self.unready += 1
        self.pending = (sessions, time.perf_counter())

    def collect(self):
        sessions, t = self.pending
        time.sleep(max(0.0, 0.001 - (time.perf_counter() - t)))
        for s in sessions:
            s.in_flight = False
        self.pending = None

    def close(self):
        pass


class FakePool:
    n_seq = 1

    def frame(self, w, h, k, i):
        return None, None


def test_admission_slices_prepare_both_graph_sets_before_frames(monkeypatch):
    monkeypatch.setattr(S, "Session", FakeSession)
    FakeSession.made = []
    srv = serve.Server.__new__(serve.Server)
    srv.lib = serve._lib.load()
    srv.pool, srv.batch, srv.stream = FakePool(), FakeBatch(), None
    srv.batches = [srv.batch]
    srv.budget, srv.max_batch, srv.frame_cost_ms, srv.load_max = 1e15, 256, None, 1.15
    clients = serve.make_clients(3, 21, rate=60.0, median_life=0.6, horizon=1.0)
    for c in clients:
        c.width, c.height = 160, 120
    n_arrivals = sum(c.t_arrive > 0 for c in clients)
    st = srv.run(clients, 1.5)
    assert n_arrivals >= 2
    assert st["admitted"] >= 3 + n_arrivals - 1
    assert srv.batch.unready == 0                       # no frame before both graph sets
    assert st["frames"] > 50 and max(srv.batch.sizes) >= 2
    live = [s for s in FakeSession.made if s.steps]
    assert len(live) >= st["admitted"] - 1
    for s in live:
        assert s.closed
        # a session admitted during the run captured one graph per slice,
        # the shared set first, then the alone set
        caps = [c for c in s.calls if c[0] == 1]
        if caps:
            flags = [shared for _, shared in caps]
            assert flags == sorted(flags, reverse=True)


def test_two_steps_in_flight(monkeypatch):
    monkeypatch.setattr(S, "Session", FakeSession)
    FakeSession.made = []
    srv = serve.Server.__new__(serve.Server)
    srv.lib = serve._lib.load()
    srv.pool, srv.stream = FakePool(), None
    srv.batches = [FakeBatch(), FakeBatch()]
    srv.batch = srv.batches[0]
    srv.budget, srv.max_batch, srv.frame_cost_ms, srv.load_max = 1e15, 4, None, 1.15
    clients = serve.make_clients(8, 5, rate=120.0, median_life=0.5, horizon=1.0)
    for c in clients:
        c.width, c.height = 160, 120
    st = srv.run(clients, 1.5)
    assert st["frames"] > 100
    assert sum(len(b.sizes) for b in srv.batches) == st["steps"]
    assert all(b.sizes for b in srv.batches)            # both batches took steps
    assert all(b.pending is None for b in srv.batches)
    for s in FakeSession.made:
        if s.steps:
            assert s.closed and not s.in_flight
