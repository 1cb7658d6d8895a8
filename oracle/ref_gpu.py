"""ORACLE — test and benchmark infrastructure only.

ctypes binding of oracle/_ref/libref_circlefft.so: the reference's own GPU circle FFT
kernels (src/cuda/kernels/circlefft.cu, compiled from the reference's source by
oracle/build_ref.sh) driven the way src/cuda/circlefft_gpu.zig:46-175 drives them
(host twiddles, device buffers allocated per call, one launch per butterfly layer,
copies in and out per call). Used by the GPU tests to check those kernels against the
oracle and by bench.py to time them beside this library's transform.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(REF_DIR, "libref_circlefft.so")
CUBIN = os.path.join(REF_DIR, "circlefft.cubin")

_lib = None


def available():
    return os.path.exists(LIB) and os.path.exists(CUBIN)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("the reference GPU circle FFT is not built (oracle/build_ref.sh)")
        L = ctypes.CDLL(LIB)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        dp = ctypes.POINTER(ctypes.c_double)
        L.ref_cfft_init.argtypes = [ctypes.c_char_p]
        L.ref_cfft_init.restype = ctypes.c_int
        L.ref_cfft_twiddles.argtypes = [ctypes.c_int]
        for f in (L.ref_cfft_fft, L.ref_cfft_ifft):
            f.argtypes = [u32p, u32p, ctypes.c_uint, dp]
            f.restype = ctypes.c_int
        rc = L.ref_cfft_init(CUBIN.encode())
        if rc != 0:
            raise RuntimeError(f"ref_cfft_init failed: {rc}")
        _lib = L
    return _lib


def set_fast_twiddles(fast: bool):
    """Build the host twiddle tree by walking the coset (same values) instead of the
    reference's per-point evaluation, which takes seconds at 2^22 points."""
    lib().ref_cfft_twiddles(int(bool(fast)))


def _call(fn, x):
    x = np.ascontiguousarray(x, dtype=np.uint32)
    n = x.size
    lg = n.bit_length() - 1
    out = np.empty(n, dtype=np.uint32)
    t = (ctypes.c_double * 2)()
    u32p = ctypes.POINTER(ctypes.c_uint32)
    rc = fn(x.ctypes.data_as(u32p), out.ctypes.data_as(u32p), lg, t)
    if rc != 0:
        raise RuntimeError(f"reference GPU circle FFT failed: {rc}")
    return out, t[0], t[1]


def fft(coeffs):
    """circleFFT of one column (A-then-B coefficients -> natural-order evaluations on
    canonicHalf(lg) ++ conjugate). Returns (evals, wall ms of the call, device ms of
    its launches)."""
    return _call(lib().ref_cfft_fft, coeffs)


def ifft(evals):
    """circleIFFT of one column. Returns (coeffs, wall ms, device ms)."""
    return _call(lib().ref_cfft_ifft, evals)
