"""The multi-GPU path of bench.py is replicas only: one session per rank,
its own seed, no collective on the data path -- the process group carries
only barriers and the max-over-ranks timing.  This exercises that host
logic with two gloo ranks on the CPU (127.0.0.1 rendezvous)."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), FB_DIST_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    import rgbd_synth as synth
    r, w, _ = bench.dist_setup(world)
    bench.barrier(w)
    ms = bench.max_over_ranks(100.0 + 10.0 * r, w)       # each rank's device time
    out[r] = (r, w, ms, bench.aggregate_value(50, w, ms), synth.session_seed(2, r))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_gloo_ranks_time_as_the_slowest_and_use_their_own_seeds():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        rank, w, ms, value, seed = res[r]
        assert (rank, w) == (r, world)
        assert ms == 110.0                                   # max over ranks
        assert value == pytest.approx(50 * world / 0.110)    # whole-job frames/s
    assert res[0][4] != res[1][4]                            # replicas: independent sequences
