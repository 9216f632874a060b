"""Host logic of the served form (no GPU): the client population and the
frame pool's playback order."""
import math

import numpy as np

from fusion_b200 import serve


def test_population_is_steady_and_lifetimes_are_lognormal():
    n, horizon = 200, 60.0
    cs = serve.make_clients(n, 5, horizon=horizon)
    warm = [c for c in cs if c.t_arrive == 0.0]
    arrivals = [c for c in cs if c.t_arrive > 0.0]
    assert len(warm) == n
    mean_life = 20.0 * math.exp(0.5 ** 2 / 2)
    expected = n / mean_life * horizon                   # Poisson count, steady population
    assert abs(len(arrivals) - expected) < 4 * math.sqrt(expected)
    assert all(0 < c.t_arrive < horizon for c in arrivals)
    assert sorted(c.t_arrive for c in arrivals) == [c.t_arrive for c in arrivals]
    life = np.array([c.lifetime for c in cs])
    assert abs(np.median(life) / 20.0 - 1) < 0.15
    assert set((c.width, c.height) for c in cs) == set(serve.RESOLUTIONS)
    v = np.array([c.voxel for c in cs])
    assert v.min() >= 0.004 and v.max() <= 0.020


def test_pool_plays_forwards_then_backwards():
    class P(serve.FramePool):
        def __init__(self):
            self.n_frames = 4
            self.seq = {(1, 1, 0): (np.arange(4), np.arange(4))}
            self.n_seq = 1
    p = P()
    order = [int(p.frame(1, 1, 0, i)[0]) for i in range(10)]
    assert order == [0, 1, 2, 3, 2, 1, 0, 1, 2, 3]


def test_sequence_seeds_are_deterministic_and_near():
    a = serve.sequence_seeds(7, 3)
    b = serve.sequence_seeds(7, 3)
    assert a == b and len(a) == 3 and len(set(a)) == 3
