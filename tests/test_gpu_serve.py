"""The served form's request loop on the GPU: admission by the HBM budget
(clients beyond it wait in the queue until departures free memory), every
arrived frame fused, latency statistics reported."""
import pytest

pytestmark = pytest.mark.gpu

pytest.importorskip("torch")


def test_budget_admission_and_continuous_batching():
    from fusion_b200 import serve
    pool = serve.FramePool(serve.sequence_seeds(7, 2), 12)
    cs = serve.make_clients(4, 11, horizon=0.0)
    for c in cs:                                   # four small sessions, short lives
        c.width, c.height, c.voxel, c.lifetime = 160, 120, 0.012, 0.6
    srv = serve.Server(pool, budget_bytes=0.0, mode=0)
    need = srv._need(cs[0])
    srv.budget = 2.5 * need                        # room for two sessions at a time
    st = srv.run(cs, 2.5)
    srv.close()
    assert st["admitted"] == 4                     # the two queued ones got in after departures
    assert st["queued"] == 2
    assert st["peak_reserved_bytes"] <= srv.budget
    assert st["frames"] > 30 and st["backlog_frames_at_end"] == 0
    assert st["latency_ms"]["p50"] > 0


def test_calibrated_load_admission():
    """Per-frame costs measured by batch steps; with the admitted GPU load
    capped, clients beyond the cap wait in the queue and are admitted as
    others leave, and the admitted load never passes the cap."""
    from fusion_b200 import serve
    pool = serve.FramePool(serve.sequence_seeds(7, 2), 12)
    srv = serve.Server(pool, budget_bytes=120e9, mode=0)
    cost = srv.calibrate(resolutions=[(160, 120), (320, 240)], sessions=2, steps=2, warmup=1)
    print("per-frame cost (ms):", cost)
    assert set(cost) == {(160, 120), (320, 240)}
    assert all(0.0 < v < 50.0 for v in cost.values())
    cs = serve.make_clients(6, 12, horizon=0.0)
    for c in cs:
        c.width, c.height, c.voxel, c.lifetime = 160, 120, 0.012, 0.6
    per = 30.0 * cost[(160, 120)]                  # GPU ms per second of one client
    srv.load_max = 2.5 * per / 1000.0              # room for two clients at a time
    st = srv.run(cs, 2.5)
    srv.close()
    print(st["admission"], st["admitted"], st["queued"])
    assert st["admitted"] == 6 and st["queued"] == 4
    assert st["admission"]["peak_admitted_load"] <= srv.load_max + 1e-12
    assert st["frames"] > 30 and st["backlog_frames_at_end"] == 0
