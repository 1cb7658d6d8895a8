"""GPU circle FFT / IFFT bit-exact against the oracle (src/cuda/circlefft_test.zig:67-108
checks log_size 3..16; this covers every size from 2 points up to 2^18)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 2**31 - 1


@pytest.mark.parametrize("log_n", list(range(1, 19)))
def test_circle_fft_matches_oracle(orc, log_n):
    from zs_b200 import native
    rng = np.random.default_rng(1000 + log_n)
    coeffs = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    assert np.array_equal(native.circle_fft(coeffs), orc.circle_fft(coeffs))
    evals = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    assert np.array_equal(native.circle_ifft(evals), orc.circle_ifft(evals))


def test_circle_fft_many_columns(orc):
    from zs_b200 import native
    rng = np.random.default_rng(5)
    x = rng.integers(0, P, (5, 1 << 12), dtype=np.uint32)
    got = native.circle_fft(x)
    for c in range(5):
        assert np.array_equal(got[c], orc.circle_fft(x[c]))
    back = native.circle_ifft(got)
    assert np.array_equal(back, x)


def test_circle_fft_edge_values(orc):
    from zs_b200 import native
    for fill in (0, 1, P - 1):
        x = np.full(1 << 11, fill, dtype=np.uint32)
        assert np.array_equal(native.circle_fft(x), orc.circle_fft(x))
        assert np.array_equal(native.circle_ifft(x), orc.circle_ifft(x))


def test_circle_fft_known_functions(orc):
    # circle.zig:403-453
    from zs_b200 import native
    xs, ys = orc.circle_domain(3)
    c = np.zeros(8, dtype=np.uint32)
    c[1] = 1
    assert np.array_equal(native.circle_fft(c), xs)
    c = np.zeros(8, dtype=np.uint32)
    c[4] = 3
    assert np.array_equal(native.circle_fft(c), (ys.astype(np.uint64) * 3 % P).astype(np.uint32))
