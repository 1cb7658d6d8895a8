"""Host logic behind the bench workloads (CPU): the seeded generators, the Fibonacci
trace against its recurrence, the job mixes of the batch and served streams, their
split over replicas, and the Poisson arrivals and percentiles of the serving loop."""
import numpy as np
import pytest

from zs_b200 import serving
from zs_b200 import workload as wl

P = wl.P


def test_splitmix64_known_outputs():
    # SplitMix64 from state 0: the published first outputs of the generator
    z = wl.splitmix64(0, 3)
    assert [int(v) for v in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_m31_range_and_determinism():
    a = wl.uniform_m31(7, 5000)
    assert a.dtype == np.uint32 and a.size == 5000
    assert int(a.max()) < P
    assert np.array_equal(a, wl.uniform_m31(7, 5000))
    assert not np.array_equal(a, wl.uniform_m31(8, 5000))
    assert np.array_equal(wl.uniform_m31(7, 100), a[:100])


@pytest.mark.parametrize("n,a0,a1", [(1, 0, 1), (2, 5, 7), (1000, 0, 1), (3000, 1, P - 1), (5000, P - 2, 3)])
def test_fib_trace_matches_recurrence(n, a0, a1):
    tr = wl.fib_trace(n, a0, a1)
    a, b = tr[0][:, 0].astype(np.int64), tr[1][:, 0].astype(np.int64)
    x, y = a0 % P, a1 % P
    for i in range(n):
        assert (a[i], b[i]) == (x, y), i
        x, y = y, (x + y) % P
    for col in tr:
        assert not col[:, 1:].any()


def test_batch_shapes_mix_and_range():
    shapes = wl.batch_shapes(512)
    assert shapes == wl.batch_shapes(512)
    assert len(shapes) == 512
    assert {s[0] for s in shapes} == {wl.AIR_SEEDED_FIB, wl.AIR_RESCUE_STACKED}
    fib = sum(1 for s in shapes if s[0] == wl.AIR_SEEDED_FIB)
    assert 200 < fib < 312
    assert all(10 <= s[1] <= 20 for s in shapes)
    assert {s[1] for s in shapes} == set(range(10, 21))
    assert len({s[3] for s in shapes}) == 512


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_batch_split_over_replicas_covers_every_job_once(world):
    shapes = wl.batch_shapes(100)
    parts = [shapes[r::world] for r in range(world)]
    assert sorted(x for p in parts for x in p) == sorted(shapes)
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_serve_shapes_geometric_sizes():
    shapes = wl.serve_shapes(4000)
    logs = np.array([s[1] for s in shapes])
    assert logs.min() >= 12 and logs.max() <= 22
    # geometric(0.5) over 12..22: about half at 12, a quarter at 13
    assert 0.45 < np.mean(logs == 12) < 0.55
    assert 0.2 < np.mean(logs == 13) < 0.3
    fib = np.mean([s[0] == wl.AIR_SEEDED_FIB for s in shapes])
    assert 0.45 < fib < 0.55
    assert len({s[3] for s in shapes}) == 4000


def test_poisson_arrivals_rate_and_order():
    t = serving.poisson_arrivals(400.0, 5.0, seed=1)
    assert all(0 < x < 5.0 for x in t)
    assert all(b > a for a, b in zip(t, t[1:]))
    assert 1800 < len(t) < 2200  # mean 2000, sd ~45
    gaps = np.diff(t)
    assert abs(gaps.mean() - 1 / 400) < 0.1 / 400
    assert t == serving.poisson_arrivals(400.0, 5.0, seed=1)


def test_percentile():
    assert np.isnan(serving.percentile([], 50))
    v = list(range(1, 101))
    assert serving.percentile(v, 50) == pytest.approx(50.5)
    assert serving.percentile(v, 99) == pytest.approx(99.01)
    assert serving.percentile([3.0], 99) == 3.0
