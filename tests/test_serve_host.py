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


def test_admission_by_memory_and_gpu_load():
    class C:
        def __init__(self, w, h, rate=30.0):
            self.width, self.height, self.rate = w, h, rate

    need = {(640, 480): 4e9, (320, 240): 1e9, (160, 120): 0.25e9}
    cost = {(640, 480): 0.5, (320, 240): 0.2, (160, 120): 0.05}
    a = serve.Admission(20e9, lambda c: need[(c.width, c.height)], cost, load_max=0.5)
    big = [C(640, 480) for _ in range(5)]
    # GPU load: 30 Hz x 0.5 ms = 15 ms per second each; 33 fit under 500 ms/s,
    # but memory admits 5 of 4 GB in 20 GB
    for c in big[:5]:
        assert a.fits(c)
        a.take(c)
    assert not a.fits(C(640, 480)) and not a.fits(C(320, 240))
    a.release(big[0])
    assert a.fits(C(320, 240))
    # load-bound: small sessions until 500 ms/s of GPU time per second
    b = serve.Admission(1e15, lambda c: 1.0, cost, load_max=0.5)
    n = 0
    while b.fits(C(160, 120)):
        b.take(C(160, 120))
        n += 1
    assert n == int(500 / (30 * 0.05) + 1e-9)
    assert abs(b.peak_load - n * 1.5) < 1e-9
    # without frame costs only memory counts
    m = serve.Admission(10.0, lambda c: 1.0)
    for _ in range(10):
        m.take(C(640, 480))
    assert not m.fits(C(160, 120)) and m.load == 0.0
