"""The reference's own GPU circle FFT kernels (src/cuda/kernels/circlefft.cu, built from
the reference's source for sm_100a into oracle/_ref/ and driven as
src/cuda/circlefft_gpu.zig:46-175 drives them) against the oracle and against this
library's transform, at the sizes src/cuda/circlefft_test.zig:67-108 checks (log 3..16)
and at 2^20. These kernels are the bar the library's circle FFT is timed against; the
test shows the bar computes the same values."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _ref():
    import ref_gpu
    if not ref_gpu.available():
        pytest.skip("oracle/_ref not built: the reference tree was absent when build() ran")
    ref_gpu.set_fast_twiddles(True)
    return ref_gpu


@pytest.mark.parametrize("log_n", [3, 4, 5, 8, 11, 12, 16, 20])
def test_reference_gpu_fft_matches_oracle_and_library(orc, log_n):
    from zs_b200 import native
    ref = _ref()
    rng = np.random.default_rng(4000 + log_n)
    coeffs = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    got, _, _ = ref.fft(coeffs)
    assert np.array_equal(got, orc.circle_fft(coeffs))
    assert np.array_equal(got, native.circle_fft(coeffs))
    evals = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    back, _, _ = ref.ifft(evals)
    assert np.array_equal(back, orc.circle_ifft(evals))
    assert np.array_equal(back, native.circle_ifft(evals))


def test_reference_gpu_faithful_twiddles(orc):
    """The per-point twiddle evaluation the reference uses gives the same transform."""
    ref = _ref()
    rng = np.random.default_rng(9)
    coeffs = rng.integers(0, P, 1 << 10, dtype=np.uint32)
    ref.set_fast_twiddles(False)
    try:
        got, _, _ = ref.fft(coeffs)
    finally:
        ref.set_fast_twiddles(True)
    assert np.array_equal(got, orc.circle_fft(coeffs))
