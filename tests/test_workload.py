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


def test_ml_linear_workload():
    """The linear-layer trace: W and inputs in [0, 2^16), y = W x mod p on the input
    rows, the input table on the other rows, the last row a table row."""
    tr, pre, pi = wl.ml_linear(6)
    D, n = wl.ML_DIM, 64
    X = np.stack([tr[l][:, 0] for l in range(D)], axis=1)
    Y = np.stack([tr[D + k][:, 0] for k in range(D)], axis=1)
    Pm = np.stack([pre[l][:, 0] for l in range(D)], axis=1)
    sel = tr[2 * D][:, 0]
    W = wl.uniform_below(wl.SEED_ML_LINEAR, D * D, 1 << 16).reshape(D, D)
    assert W.max() < (1 << 16) and X.max() < (1 << 16)
    assert (sel[: n // 2] == 1).all() and (sel[n // 2:] == 0).all() and sel[-1] == 0
    assert np.array_equal(Y, (X.astype(np.uint64) @ W.T.astype(np.uint64)) % wl.P)
    assert np.array_equal(Pm[n // 2:], X[: n // 2]) and not Pm[: n // 2].any() and not X[n // 2:].any()
    assert len(pi) == 8 + 16 * D * D
    for c in tr + pre:
        assert c.shape == (n, 4) and not c[:, 1:].any()


def test_serve_mix_includes_the_linear_layer():
    shapes = wl.serve_shapes(4000)
    airs = np.array([s[0] for s in shapes])
    assert 0.25 < np.mean(airs == wl.AIR_RESCUE_STACKED) < 0.35
    assert 0.15 < np.mean(airs == wl.AIR_ML_LINEAR) < 0.25
    assert max(s[1] for s in shapes if s[0] == wl.AIR_ML_LINEAR) <= wl.ML_LINEAR_MAX_LOG
