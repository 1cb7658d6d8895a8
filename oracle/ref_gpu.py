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


# ---- the reference's GPU sum-check round kernels (src/cuda/kernels/sumcheck.cu) ----------

SC_LIB = os.path.join(REF_DIR, "libref_sumcheck.so")
SC_CUBIN = os.path.join(REF_DIR, "sumcheck.cubin")
_sc_lib = None


def sumcheck_available():
    return os.path.exists(SC_LIB) and os.path.exists(SC_CUBIN)


def sumcheck_lib():
    global _sc_lib
    if _sc_lib is None:
        if not sumcheck_available():
            raise RuntimeError("the reference GPU sum-check kernels are not built (oracle/build_ref.sh)")
        L = ctypes.CDLL(SC_LIB)
        L.ref_sc_init.argtypes = [ctypes.c_char_p]
        L.ref_sc_init.restype = ctypes.c_int
        sz = ctypes.c_size_t
        L.ref_sc_values.argtypes = [ctypes.c_int, ctypes.c_char_p, sz, sz, ctypes.c_char_p, sz, ctypes.c_void_p, sz,
                                    ctypes.c_void_p, sz, sz, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        L.ref_sc_values.restype = ctypes.c_int
        rc = L.ref_sc_init(SC_CUBIN.encode())
        if rc != 0:
            raise RuntimeError(f"ref_sc_init failed: {rc}")
        _sc_lib = L
    return _sc_lib


def sumcheck_values(wide, cur_flat: bytes, length, m, coeffs: bytes, indices, offsets, dmax, half):
    """One round through the reference's own kernel, driven as src/cuda/sumcheck_gpu.zig
    drives it (buffers allocated and copied per call). Returns (values bytes, wall ms of
    the call, device ms of the launch)."""
    es = 16 if wide else 1
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    out = ctypes.create_string_buffer((dmax + 1) * es)
    t = (ctypes.c_double * 2)()
    rc = sumcheck_lib().ref_sc_values(int(bool(wide)), bytes(cur_flat), length, m, bytes(coeffs),
                                      len(coeffs) // es, idx.ctypes.data, idx.size, off.ctypes.data, dmax, half,
                                      out, t)
    if rc != 0:
        raise RuntimeError(f"reference GPU sum-check round failed: {rc}")
    return out.raw, t[0], t[1]
