"""ctypes binding of ``libzs_b200.so`` (the C ABI in include/zs_m31.h).

The GPU library is the only implementation behind these calls: there is no CPU
fallback, and loading fails loudly when the library has not been built.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzs_b200.so")
_lib = None

u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)

ERRORS = {-1: "generic error", -2: "malformed input", -3: "out of memory", -4: "protocol error",
          -5: "device error"}


class ZsError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed: {code} ({ERRORS.get(code, 'unknown')})")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `make -C zig-stark_b200` "
                              "(or __graft_entry__.build()) first")
        L = ctypes.CDLL(LIB_PATH)
        L.zs_version.restype = ctypes.c_char_p
        L.zs_m31_circle_fft.argtypes = [u32p, ctypes.c_uint32] + [ctypes.c_uint32] * 5 + [u32p]
        L.zs_m31_circle_ifft.argtypes = [u32p, ctypes.c_uint32] + [ctypes.c_uint32] * 5 + [u32p]
        L.zs_m31_commit_plan_create.argtypes = [ctypes.c_uint32] * 4 + [ctypes.POINTER(ctypes.c_void_p)]
        L.zs_m31_commit_plan_destroy.argtypes = [ctypes.c_void_p]
        L.zs_m31_commit_plan_destroy.restype = None
        L.zs_m31_commit_plan_set_challenges.argtypes = [ctypes.c_void_p, u32p, u32p]
        L.zs_m31_commit_plan_trace_buffer.argtypes = [ctypes.c_void_p]
        L.zs_m31_commit_plan_trace_buffer.restype = ctypes.c_void_p
        L.zs_m31_commit_plan_upload.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.zs_m31_commit_plan_run_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.zs_m31_commit_plan_run_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.zs_m31_commit_plan_run_phase.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                                    ctypes.c_void_p]
        L.zs_m31_commit_plan_results.argtypes = [ctypes.c_void_p, ctypes.c_void_p, u8p, u8p, u32p]
        L.zs_m31_commit_plan_copy_lde.argtypes = [ctypes.c_void_p, u32p]
        L.zs_m31_commit_plan_copy_layer.argtypes = [ctypes.c_void_p, ctypes.c_uint32, u32p]
        L.zs_m31_commit_plan_launches.argtypes = [ctypes.c_void_p]
        L.zs_m31_commit_plan_launches.restype = ctypes.c_uint32
        L.zs_m31_circle_commit.argtypes = [u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u32p, u32p,
                                           ctypes.c_uint32, u8p, u8p, u32p]
        L.zs_m31_circle_lde_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
        _lib = L
    return _lib


def check(rc, what):
    if rc != 0:
        raise ZsError(rc, what)


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(u32p)


def version():
    return lib().zs_version().decode()


# ---------------------------------------------------------------------------
# circle FFT (src/cuda/circlefft_gpu.zig:46-175)
# ---------------------------------------------------------------------------

P = 2147483647


def _pt_add(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def _pt_mul(pt, k):
    r = (1, 0)
    while k:
        if k & 1:
            r = _pt_add(r, pt)
        pt = _pt_add(pt, pt)
        k >>= 1
    return r


def canonic_half_coset(log_size):
    """CircleCoset.canonicHalf(log_size) (coset.zig:59-65) as (offset, step, log_half)."""
    gen_neg = (1268011823, P - 2)
    return _pt_mul(gen_neg, 1 << (30 - log_size)), _pt_mul(gen_neg, 1 << (32 - log_size)), log_size - 1


def circle_fft(coeffs, half_coset=None):
    """circleFFT: A-then-B coefficients -> natural-order evaluations on
    half_coset ++ conjugate. `coeffs` is (n,) or (columns, n); `half_coset` =
    (offset, step, log_half), default canonicHalf(log2 n)."""
    return _circle(coeffs, half_coset, inverse=False)


def circle_ifft(evals, half_coset=None):
    """circleIFFT: natural-order evaluations -> A-then-B coefficients."""
    return _circle(evals, half_coset, inverse=True)


def _circle(x, half_coset, inverse):
    x, p = _u32(x)
    n = x.shape[-1]
    cols = x.size // n
    log_n = n.bit_length() - 1
    if (1 << log_n) != n or n < 2:
        raise ValueError("transform length must be a power of two >= 2")
    if half_coset is None:
        half_coset = canonic_half_coset(log_n)
    (ox, oy), (sx, sy), log_half = half_coset
    if log_half + 1 != log_n:
        raise ValueError("half coset size does not match the transform length")
    out = np.empty_like(x)
    fn = lib().zs_m31_circle_ifft if inverse else lib().zs_m31_circle_fft
    check(fn(p, cols, ox, oy, sx, sy, log_half, out.ctypes.data_as(u32p)),
          "zs_m31_circle_ifft" if inverse else "zs_m31_circle_fft")
    return out


# ---------------------------------------------------------------------------
# circle commit workload
# ---------------------------------------------------------------------------

class CommitPlan:
    """Device-resident plan of the circle commit workload (zs_m31_commit_plan_*)."""

    def __init__(self, n_columns, log_rows, log_blowup, n_folds):
        self.n_columns, self.log_rows, self.log_blowup, self.n_folds = n_columns, log_rows, log_blowup, n_folds
        h = ctypes.c_void_p()
        check(lib().zs_m31_commit_plan_create(n_columns, log_rows, log_blowup, n_folds, ctypes.byref(h)),
              "zs_m31_commit_plan_create")
        self._h = h

    def close(self):
        if self._h:
            lib().zs_m31_commit_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_challenges(self, gammas, alphas):
        g, pg = _u32(gammas)
        a, pa = _u32(alphas if self.n_folds else np.zeros(4, np.uint32))
        check(lib().zs_m31_commit_plan_set_challenges(self._h, pg, pa), "zs_m31_commit_plan_set_challenges")

    def trace_ptr(self):
        return lib().zs_m31_commit_plan_trace_buffer(self._h)

    def upload(self, trace, stream=None):
        """trace: host array (n_columns, 2^log_rows); pinned memory makes the copy asynchronous."""
        if isinstance(trace, np.ndarray):
            trace = np.ascontiguousarray(trace, dtype=np.uint32)
            ptr = trace.ctypes.data
        else:
            ptr = int(trace)
        check(lib().zs_m31_commit_plan_upload(self._h, ctypes.c_void_p(ptr), ctypes.c_void_p(stream or 0)),
              "zs_m31_commit_plan_upload")

    def run(self, d_trace=None, stream=None):
        check(lib().zs_m31_commit_plan_run_device(self._h, ctypes.c_void_p(d_trace or 0),
                                                  ctypes.c_void_p(stream or 0)), "zs_m31_commit_plan_run_device")

    def run_host(self, host_ptr, stream=None):
        """The step from a pinned host trace (pointer), its upload overlapped with the LDE."""
        check(lib().zs_m31_commit_plan_run_host(self._h, ctypes.c_void_p(int(host_ptr)), ctypes.c_void_p(stream or 0)),
              "zs_m31_commit_plan_run_host")

    PHASES = ("lde", "row_tree", "folds")

    def run_phase(self, phase, d_trace=None, stream=None):
        check(lib().zs_m31_commit_plan_run_phase(self._h, phase, ctypes.c_void_p(d_trace or 0),
                                                 ctypes.c_void_p(stream or 0)), "zs_m31_commit_plan_run_phase")

    def results(self, stream=None):
        root = (ctypes.c_uint8 * 32)()
        layer_roots = np.zeros((self.n_folds, 32), dtype=np.uint8)
        final = np.zeros((1 << (self.log_rows + self.log_blowup - self.n_folds), 4), dtype=np.uint32)
        check(lib().zs_m31_commit_plan_results(self._h, ctypes.c_void_p(stream or 0), root,
                                               layer_roots.ctypes.data_as(u8p), final.ctypes.data_as(u32p)),
              "zs_m31_commit_plan_results")
        return {"lde_root": bytes(root), "layer_roots": layer_roots, "final_layer": final}

    def lde(self):
        out = np.zeros((self.n_columns, 1 << (self.log_rows + self.log_blowup)), dtype=np.uint32)
        check(lib().zs_m31_commit_plan_copy_lde(self._h, out.ctypes.data_as(u32p)), "zs_m31_commit_plan_copy_lde")
        return out

    def layer(self, i):
        out = np.zeros((1 << (self.log_rows + self.log_blowup - i), 4), dtype=np.uint32)
        check(lib().zs_m31_commit_plan_copy_layer(self._h, i, out.ctypes.data_as(u32p)),
              "zs_m31_commit_plan_copy_layer")
        return out

    def launches(self):
        return int(lib().zs_m31_commit_plan_launches(self._h))


def circle_commit(trace, log_blowup, gammas, alphas):
    """One-shot host-buffer call (zs_m31_circle_commit)."""
    trace, pt = _u32(trace)
    n_cols, n = trace.shape
    log_rows = n.bit_length() - 1
    g, pg = _u32(gammas)
    a, pa = _u32(alphas)
    n_folds = a.size // 4
    root = (ctypes.c_uint8 * 32)()
    layer_roots = np.zeros((max(n_folds, 1), 32), dtype=np.uint8)
    final = np.zeros((1 << (log_rows + log_blowup - n_folds), 4), dtype=np.uint32)
    check(lib().zs_m31_circle_commit(pt, n_cols, log_rows, log_blowup, pg, pa, n_folds, root,
                                     layer_roots.ctypes.data_as(u8p), final.ctypes.data_as(u32p)),
          "zs_m31_circle_commit")
    return {"lde_root": bytes(root), "layer_roots": layer_roots[:n_folds], "final_layer": final}


def circle_lde_noalloc(d_in, d_out, n_columns, log_rows, log_blowup, stream=None):
    """zs_m31_circle_lde_noalloc on caller-owned device buffers (device pointers as
    ints); returns the C ABI status code."""
    return int(lib().zs_m31_circle_lde_noalloc(ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), n_columns, log_rows,
                                               log_blowup, ctypes.c_void_p(stream or 0)))


# ---------------------------------------------------------------------------
# prover (zs_m31_prove)
# ---------------------------------------------------------------------------

_libc = ctypes.CDLL(None)
_libc.malloc.restype = ctypes.c_void_p
_libc.malloc.argtypes = [ctypes.c_size_t]
_libc.free.restype = None
_libc.free.argtypes = [ctypes.c_void_p]
_ALLOC_T = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)
_FREE_T = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)


class HostAllocator(ctypes.Structure):
    """zs_host_allocator (zig-capi.h:35-39) backed by the C library's malloc/free."""
    _fields_ = [("ctx", ctypes.c_void_p), ("alloc", _ALLOC_T), ("free", _FREE_T)]


_ALLOC = _ALLOC_T(lambda ctx, size: _libc.malloc(size))
_FREE = _FREE_T(lambda ctx, ptr, size: _libc.free(ptr))
HOST = HostAllocator(None, _ALLOC, _FREE)


def _bind_prove():
    L = lib()
    if not getattr(L, "_prove_bound", False):
        L.zs_m31_prove.argtypes = [HostAllocator, ctypes.c_uint32] + [ctypes.c_char_p, ctypes.c_size_t] * 5 + \
            [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]
        L.zs_free.argtypes = [HostAllocator, ctypes.c_void_p, ctypes.c_size_t]
        L.zs_free.restype = None
        L._prove_bound = True
    return L


def prove(air_id, params, public_inputs, trace, preprocessed=b"", channel_sep=b""):
    """GenericStark(Air).proveWithPreprocessed on the GPU; returns the serialized proof.

    params: wire StarkParams bytes (or wire.StarkParams); trace / preprocessed: wire
    []const []const QM31 bytes (or lists of (n, 4) uint32 arrays)."""
    from . import wire
    if not isinstance(params, (bytes, bytearray)):
        params = params.encode()
    if not isinstance(trace, (bytes, bytearray)):
        trace = wire.columns(trace)
    if not isinstance(preprocessed, (bytes, bytearray)):
        preprocessed = wire.columns(preprocessed)
    L = _bind_prove()
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    check(L.zs_m31_prove(HOST, air_id, params, len(params), public_inputs, len(public_inputs), preprocessed,
                         len(preprocessed), trace, len(trace), channel_sep, len(channel_sep), ctypes.byref(out),
                         ctypes.byref(n)), "zs_m31_prove")
    data = ctypes.string_at(out.value, n.value)
    L.zs_free(HOST, out, n.value)
    return data


class Context:
    """A device context (zs_m31_ctx_*): a CUDA device ordinal and a stream of its own.
    prove() is `prove` run on that device and stream; calls on one context run one at a
    time, calls on distinct contexts concurrently."""

    def __init__(self, device=0):
        L = _bind_prove()
        if not getattr(L, "_ctx_bound", False):
            L.zs_m31_ctx_create.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
            L.zs_m31_ctx_destroy.argtypes = [ctypes.c_void_p]
            L.zs_m31_ctx_destroy.restype = None
            L.zs_m31_ctx_device.argtypes = [ctypes.c_void_p]
            L.zs_m31_prove_ctx.argtypes = [ctypes.c_void_p] + L.zs_m31_prove.argtypes
            L._ctx_bound = True
        self._L = L
        self._h = None
        h = ctypes.c_void_p()
        check(L.zs_m31_ctx_create(device, ctypes.byref(h)), "zs_m31_ctx_create")
        self._h = h

    @property
    def device(self):
        return self._L.zs_m31_ctx_device(self._h)

    def prove(self, air_id, params, public_inputs, trace, preprocessed=b"", channel_sep=b""):
        from . import wire
        if not isinstance(params, (bytes, bytearray)):
            params = params.encode()
        if not isinstance(trace, (bytes, bytearray)):
            trace = wire.columns(trace)
        if not isinstance(preprocessed, (bytes, bytearray)):
            preprocessed = wire.columns(preprocessed)
        out = ctypes.c_void_p()
        n = ctypes.c_size_t()
        check(self._L.zs_m31_prove_ctx(self._h, HOST, air_id, params, len(params), public_inputs,
                                       len(public_inputs), preprocessed, len(preprocessed), trace, len(trace),
                                       channel_sep, len(channel_sep), ctypes.byref(out), ctypes.byref(n)),
              "zs_m31_prove_ctx")
        data = ctypes.string_at(out.value, n.value)
        self._L.zs_free(HOST, out, n.value)
        return data

    def close(self):
        if self._h:
            self._L.zs_m31_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def verify(air_id, params, public_inputs, proof, channel_sep=b""):
    """GenericStark(Air).verify (zs_m31_verify, host-side); returns True / False."""
    if not isinstance(params, (bytes, bytearray)):
        params = params.encode()
    L = _bind_prove()
    if not getattr(L, "_verify_bound", False):
        L.zs_m31_verify.argtypes = [HostAllocator, ctypes.c_uint32] + [ctypes.c_char_p, ctypes.c_size_t] * 4 + \
            [ctypes.POINTER(ctypes.c_int)]
        L._verify_bound = True
    ok = ctypes.c_int()
    check(L.zs_m31_verify(HOST, air_id, params, len(params), public_inputs, len(public_inputs), proof, len(proof),
                          channel_sep, len(channel_sep), ctypes.byref(ok)), "zs_m31_verify")
    return bool(ok.value)


class VerifyJob(ctypes.Structure):
    """zs_m31_verify_job: the arguments of one zs_m31_verify call."""
    _fields_ = [("air_id", ctypes.c_uint32),
                ("params", ctypes.c_char_p), ("params_len", ctypes.c_size_t),
                ("public_inputs", ctypes.c_char_p), ("public_inputs_len", ctypes.c_size_t),
                ("proof", ctypes.c_char_p), ("proof_len", ctypes.c_size_t),
                ("channel_sep", ctypes.c_char_p), ("channel_sep_len", ctypes.c_size_t)]


def verify_batch(jobs, threads=0):
    """zs_m31_verify_batch over (air_id, params, public_inputs, proof, channel_sep)
    tuples; returns one entry per job: True / False, or the negative status code of a
    job whose inputs could not be parsed."""
    L = _bind_prove()
    if not getattr(L, "_verify_batch_bound", False):
        L.zs_m31_verify_batch.argtypes = [ctypes.c_size_t, ctypes.POINTER(VerifyJob), ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int32)]
        L._verify_batch_bound = True
    packed = []
    for air, params, pi, proof, sep in jobs:
        if not isinstance(params, (bytes, bytearray)):
            params = params.encode()
        packed.append(VerifyJob(air, bytes(params), len(params), bytes(pi), len(pi), bytes(proof), len(proof),
                                bytes(sep), len(sep)))
    n = len(packed)
    arr = (VerifyJob * max(n, 1))(*packed)
    ok = (ctypes.c_int * max(n, 1))()
    st = (ctypes.c_int32 * max(n, 1))()
    check(L.zs_m31_verify_batch(n, arr, threads, ok, st), "zs_m31_verify_batch")
    return [bool(ok[i]) if st[i] == 0 else int(st[i]) for i in range(n)]


def commit_columns(columns, trace_log, log_blowup):
    """Per-column commitment roots (zs_m31_commit_columns); columns: wire bytes or a
    list of (2^trace_log, 4) uint32 arrays. Returns a list of 32-byte roots."""
    from . import wire
    if not isinstance(columns, (bytes, bytearray)):
        columns = wire.columns(columns)
    L = _bind_prove()
    if not getattr(L, "_commit_bound", False):
        L.zs_m31_commit_columns.argtypes = [HostAllocator, ctypes.c_uint8, ctypes.c_uint8, ctypes.c_char_p,
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p),
                                            ctypes.POINTER(ctypes.c_size_t)]
        L._commit_bound = True
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    check(L.zs_m31_commit_columns(HOST, trace_log, log_blowup, columns, len(columns), ctypes.byref(out),
                                  ctypes.byref(n)), "zs_m31_commit_columns")
    data = ctypes.string_at(out.value, n.value)
    L.zs_free(HOST, out, n.value)
    r = wire.Reader(data)
    roots = r.digests()
    r.end()
    return roots


# ---------------------------------------------------------------------------
# batched and served proving (zs_m31_prove_batch, zs_m31_server_*)
# ---------------------------------------------------------------------------

class Job(ctypes.Structure):
    """zs_m31_job: the arguments of one zs_m31_prove call."""
    _fields_ = [("air_id", ctypes.c_uint32),
                ("params", ctypes.c_char_p), ("params_len", ctypes.c_size_t),
                ("public_inputs", ctypes.c_char_p), ("public_inputs_len", ctypes.c_size_t),
                ("preprocessed", ctypes.c_char_p), ("preprocessed_len", ctypes.c_size_t),
                ("trace", ctypes.c_char_p), ("trace_len", ctypes.c_size_t),
                ("channel_sep", ctypes.c_char_p), ("channel_sep_len", ctypes.c_size_t)]


class Result(ctypes.Structure):
    """zs_m31_result: a proof in host memory and its status (1 = pending)."""
    _fields_ = [("proof", ctypes.c_void_p), ("len", ctypes.c_size_t), ("status", ctypes.c_int32)]


PENDING = 1


def _job_bytes(air_id, params, public_inputs, trace, preprocessed=b"", channel_sep=b""):
    from . import wire
    if not isinstance(params, (bytes, bytearray)):
        params = params.encode()
    if not isinstance(trace, (bytes, bytearray)):
        trace = wire.columns(trace)
    if not isinstance(preprocessed, (bytes, bytearray)):
        preprocessed = wire.columns(preprocessed)
    return (int(air_id), bytes(params), bytes(public_inputs), bytes(preprocessed), bytes(trace), bytes(channel_sep))


def _make_job(b):
    air_id, params, pi, pre, trace, sep = b
    return Job(air_id, params, len(params), pi, len(pi), pre, len(pre), trace, len(trace), sep, len(sep))


def _bind_batch():
    L = _bind_prove()
    if not getattr(L, "_batch_bound", False):
        L.zs_m31_prove_batch.argtypes = [HostAllocator, ctypes.c_size_t, ctypes.POINTER(Job), ctypes.c_uint32,
                                         ctypes.c_uint64, ctypes.POINTER(Result)]
        L.zs_m31_server_create.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
        L.zs_m31_server_destroy.argtypes = [ctypes.c_void_p]
        L.zs_m31_server_destroy.restype = None
        L.zs_m31_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.POINTER(ctypes.c_uint64)]
        L.zs_m31_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, HostAllocator,
                                         ctypes.POINTER(Result), ctypes.POINTER(ctypes.c_double)]
        L._batch_bound = True
    return L


def _take(L, res):
    """Copies a finished result's proof out of the host allocator's buffer and frees it."""
    if res.status != 0:
        return None
    data = ctypes.string_at(res.proof, res.len)
    L.zs_free(HOST, res.proof, res.len)
    return data


def prove_batch(jobs, concurrency=8, hbm_budget=0):
    """Proves independent traces together (zs_m31_prove_batch).

    jobs: tuples or dicts of prove()'s arguments (air_id, params, public_inputs,
    trace[, preprocessed[, channel_sep]]). Returns one entry per job: the proof bytes,
    or the negative status code of a job that failed (the others still complete)."""
    packed = [_job_bytes(**j) if isinstance(j, dict) else _job_bytes(*j) for j in jobs]
    arr = (Job * max(len(packed), 1))(*[_make_job(b) for b in packed])
    res = (Result * max(len(packed), 1))()
    L = _bind_batch()
    check(L.zs_m31_prove_batch(HOST, len(packed), arr, concurrency, hbm_budget, res), "zs_m31_prove_batch")
    out = []
    for i in range(len(packed)):
        d = _take(L, res[i])
        out.append(d if d is not None else int(res[i].status))
    return out


class Server:
    """A proof server (zs_m31_server_*): submit() queues a request and returns a
    ticket; poll(ticket) returns (proof bytes or negative status, latency_ms), or None
    while the request is pending and wait is False."""

    def __init__(self, workers=8, hbm_budget=0):
        self._L = _bind_batch()
        h = ctypes.c_void_p()
        check(self._L.zs_m31_server_create(workers, hbm_budget, ctypes.byref(h)), "zs_m31_server_create")
        self._h = h

    def submit(self, air_id, params, public_inputs, trace, preprocessed=b"", channel_sep=b""):
        job = _make_job(_job_bytes(air_id, params, public_inputs, trace, preprocessed, channel_sep))
        t = ctypes.c_uint64()
        check(self._L.zs_m31_server_submit(self._h, ctypes.byref(job), ctypes.byref(t)), "zs_m31_server_submit")
        return t.value

    def poll(self, ticket, wait=True):
        res = Result()
        lat = ctypes.c_double()
        check(self._L.zs_m31_server_poll(self._h, ticket, 1 if wait else 0, HOST, ctypes.byref(res),
                                         ctypes.byref(lat)), "zs_m31_server_poll")
        if res.status == PENDING:
            return None
        d = _take(self._L, res)
        return (d if d is not None else int(res.status)), lat.value

    def close(self):
        if self._h:
            self._L.zs_m31_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _host_buffer(buf):
    """(pointer or bytes, size in bytes) of bytes-like host data or of a CPU tensor (pinned
    memory makes the host-to-device copies direct)."""
    if hasattr(buf, "data_ptr"):
        if buf.is_cuda:
            raise ZsError(-2, "binius: host tables expected")
        return buf.data_ptr(), buf.numel() * buf.element_size()
    buf = bytes(buf)
    return buf, len(buf)


def _binius_values(fn, es, cur_flat, length, m, coeffs, indices, offsets, dmax, half):
    cur, size = _host_buffer(cur_flat)
    coeffs = bytes(coeffs)
    if size != m * length * es or len(coeffs) % es:
        raise ZsError(-2, "binius values: buffer sizes")
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    if off.size != len(coeffs) // es + 1:
        raise ZsError(-2, "binius values: offsets")
    out = ctypes.create_string_buffer((dmax + 1) * es)
    check(fn(cur, length, m, coeffs, len(coeffs) // es, idx.ctypes.data_as(u32p), idx.size,
             off.ctypes.data_as(u32p), dmax, half, out, None), fn.__name__)
    return out.raw


def _bind_binius():
    L = lib()
    if not getattr(L, "_binius_bound", False):
        sz, cp, vp = ctypes.c_size_t, ctypes.c_char_p, ctypes.c_void_p
        for fn in (L.zs_binius_sumcheck_values_gf256, L.zs_binius_sumcheck_values_gf128):
            fn.argtypes = [vp, sz, sz, cp, sz, u32p, sz, u32p, sz, sz, cp, vp]
        L.zs_binius_sumcheck_values_device.argtypes = [ctypes.c_uint32, vp, sz, sz, cp, sz, u32p, sz, u32p, sz, sz,
                                                       vp, vp]
        L.zs_binius_sumcheck_fold_device.argtypes = [ctypes.c_uint32, vp, sz, sz, cp, vp, vp, vp]
        L.zs_binius_sumcheck_prove_combination.argtypes = [ctypes.c_uint32, vp, sz, sz, cp, sz, u32p, sz, u32p, cp,
                                                           sz, ctypes.c_int32, cp, cp, vp]
        L._binius_bound = True
    return L


def binius_terms(terms, es):
    """[(factor table indices, coefficient int)] -> (coefficient bytes, indices, offsets)."""
    coeffs = b"".join(int(c).to_bytes(es, "little") for _, c in terms)
    idx = np.array([f for fs, _ in terms for f in fs], dtype=np.uint32)
    off = np.zeros(len(terms) + 1, dtype=np.uint32)
    off[1:] = np.cumsum([len(fs) for fs, _ in terms])
    return coeffs, idx, off


def binius_values_device(field_bits, d_cur, length, m, terms, dmax, half, d_out, stream=None):
    """zs_binius_sumcheck_values_device on device tables (pointers as ints); asynchronous."""
    es = 1 if field_bits == 8 else 16
    coeffs, idx, off = binius_terms(terms, es)
    L = _bind_binius()
    check(L.zs_binius_sumcheck_values_device(field_bits, d_cur, length, m, coeffs, len(terms),
                                             idx.ctypes.data_as(u32p), idx.size, off.ctypes.data_as(u32p), dmax,
                                             half, d_out, stream), "zs_binius_sumcheck_values_device")


def binius_fold_device(field_bits, d_cur, length, m, r, d_next, d_scratch=None, stream=None):
    """zs_binius_sumcheck_fold_device: d_next = the fold of d_cur at r (an int)."""
    es = 1 if field_bits == 8 else 16
    L = _bind_binius()
    check(L.zs_binius_sumcheck_fold_device(field_bits, d_cur, length, m, int(r).to_bytes(es, "little"), d_next,
                                           d_scratch, stream), "zs_binius_sumcheck_fold_device")


def binius_prove_combination(field_bits, tables, k, m, terms, seed=None, stream=None):
    """Sumcheck(F).proveCombination (src/binius/sumcheck.zig:208-395) on the device:
    tables = m tables of 2^k elements (bytes or a CPU tensor, little-endian; 1 byte per
    element for field_bits 8, 16 for 128); terms = [(factor indices, coefficient int)]; seed = bytes
    for proveCombination's optional transcript seed. Returns (claimed sum bytes, rounds bytes)."""
    es = 1 if field_bits == 8 else 16
    coeffs, idx, off = binius_terms(terms, es)
    dmax = max((len(fs) for fs, _ in terms), default=0)
    claimed = ctypes.create_string_buffer(es)
    rounds = ctypes.create_string_buffer(max(1, k * (dmax + 1) * es))
    sd = b"" if seed is None else bytes(seed)
    tab, size = _host_buffer(tables)
    if size != m * (1 << k) * es:
        raise ZsError(-2, "binius prove: table size")
    L = _bind_binius()
    check(L.zs_binius_sumcheck_prove_combination(field_bits, tab, k, m, coeffs, len(terms),
                                                 idx.ctypes.data_as(u32p), idx.size, off.ctypes.data_as(u32p), sd,
                                                 len(sd), int(seed is not None), claimed, rounds, stream),
          "zs_binius_sumcheck_prove_combination")
    return claimed.raw, rounds.raw[:k * (dmax + 1) * es]


def binius_gf256_values(cur_flat, length, m, coeffs, indices, offsets, dmax, half):
    """accel.Gf256ValuesFn (src/binius/accel.zig:9-26): one sum-check round's values[t],
    t = 0..dmax, over GF(2^8) (zs_binius_sumcheck_values_gf256). cur_flat holds m tables
    of `length` bytes; term k has coefficient coeffs[k] and the factor tables
    indices[offsets[k]:offsets[k + 1]]. Returns dmax + 1 bytes."""
    L = _bind_binius()
    return _binius_values(L.zs_binius_sumcheck_values_gf256, 1, cur_flat, length, m, coeffs, indices, offsets,
                          dmax, half)


def binius_gf128_values(cur_flat, length, m, coeffs, indices, offsets, dmax, half):
    """accel.Gf128ValuesFn (src/binius/accel.zig:43-47): as binius_gf256_values over
    GF(2^128), every element 16 little-endian bytes. Returns (dmax + 1) * 16 bytes."""
    L = _bind_binius()
    return _binius_values(L.zs_binius_sumcheck_values_gf128, 16, cur_flat, length, m, coeffs, indices, offsets,
                          dmax, half)
