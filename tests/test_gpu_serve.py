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
