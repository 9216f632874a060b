"""The served form's request loop (fusion_b200/serve.py) on the host with
fakes for the sessions, the batch and the frame pool (no GPU): arrivals are
admitted in order, each session captures both sets of frame graphs (steps
of other sessions, then steps alone) one capture per admission slice before
its first frame, frames are stepped in batches of the clients with pending
frames, and departures close sessions."""
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
        self.closed = True


class FakeBatch:
    def __init__(self):
        self.sizes = []
        self.unready = 0

    def reserve(self, n):
        pass

    def step(self, sessions, frames):
        self.sizes.append(len(sessions))
        for s in sessions:
            s.steps += 1
            if s.missing[True] or s.missing[False]:
                self.unready += 1
        time.sleep(0.001)

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
