"""Host logic of the serving workload (no GPU): the seeded request stream, Poisson
arrivals and the first-come first-served recurrence used for the one-at-a-time plain
baseline."""
import numpy as np
import pytest

from gianduia_b200 import serving as S


def test_requests_are_seeded_and_cover_the_grid():
    a = S.make_requests(3000, seed=4)
    assert a == S.make_requests(3000, seed=4)
    assert a != S.make_requests(3000, seed=5)
    assert {r["scene"] for r in a} == set(S.SCENES)
    assert {r["res"] for r in a} == set(S.RESOLUTIONS)
    assert {r["spp"] for r in a} == set(S.SPPS)
    depths = {r["max_depth"] for r in a}
    assert min(depths) == S.DEPTH_MIN and max(depths) == S.DEPTH_MAX
    # uniform choices: each scene within 5 sigma of n/3
    for s in S.SCENES:
        k = sum(r["scene"] == s for r in a)
        assert abs(k - 1000) < 5 * np.sqrt(3000 * (1 / 3) * (2 / 3))
    mean = np.mean([S.samples(r) for r in a])
    assert abs(mean / S.mean_samples_per_request() - 1) < 0.1


def test_poisson_arrivals():
    t = S.poisson_arrivals(20000, rate=50.0, seed=4)
    assert np.all(np.diff(t) > 0) and t[0] > 0
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 50.0) < 5 * (1 / 50.0) / np.sqrt(20000)
    # exponential gaps: coefficient of variation 1
    assert abs(gaps.std() / gaps.mean() - 1) < 0.05
    with pytest.raises(ValueError):
        S.poisson_arrivals(3, rate=0)


def test_fifo_finish_recurrence():
    arr = np.array([0.0, 0.5, 0.6, 5.0])
    svc = np.array([1.0, 1.0, 0.1, 0.5])
    f = S.fifo_finish(arr, svc)
    assert np.allclose(f, [1.0, 2.0, 2.1, 5.5])
    # an idle server starts each job on arrival
    f2 = S.fifo_finish([0.0, 10.0], [1.0, 1.0])
    assert np.allclose(f2, [1.0, 11.0])
    with pytest.raises(ValueError):
        S.fifo_finish([0.0], [1.0, 2.0])


def test_latency_stats():
    st = S.latency_stats(np.arange(1, 101, dtype=float))
    assert st["p50"] == pytest.approx(50.5) and st["p99"] == pytest.approx(99.01)
    assert st["max"] == 100.0
