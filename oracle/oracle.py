"""ORACLE — test infrastructure only.

ctypes binding of the CPU restatement of the reference (``oracle/build/liboracle.so``).
Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg load
it, and only as the checker; the product (``zig-stark_b200``) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")
_lib = None

u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_blake3.argtypes = [ctypes.c_char_p, ctypes.c_size_t, u8p]
        L.orc_hash2.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u8p]
        L.orc_hash_qm31.argtypes = [u32p, ctypes.c_size_t, u8p]
        L.orc_hash_m31_rows.argtypes = [u32p, ctypes.c_size_t, ctypes.c_size_t, u8p]
        L.orc_m31_op.argtypes = [ctypes.c_int, u32p, u32p, u32p, ctypes.c_size_t]
        L.orc_qm31_op.argtypes = [ctypes.c_int, u32p, u32p, u32p, ctypes.c_size_t]
        L.orc_qm31_pow.argtypes = [u32p, ctypes.c_uint64, u32p]
        L.orc_qm31_root.argtypes = [ctypes.c_uint, u32p]
        L.orc_circle_generator_mul.argtypes = [ctypes.c_uint64, u32p]
        L.orc_circle_domain.argtypes = [ctypes.c_uint, u32p, u32p]
        L.orc_circle_fft.argtypes = [u32p, ctypes.c_uint, u32p, ctypes.c_int]
        L.orc_circle_ifft.argtypes = [u32p, ctypes.c_uint, u32p, ctypes.c_int]
        L.orc_circle_eval_at.argtypes = [u32p, ctypes.c_uint, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_circle_eval_at.restype = ctypes.c_uint32
        L.orc_wire_golden.restype = ctypes.c_size_t
        L.orc_binius_values.argtypes = [ctypes.c_uint, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_size_t,
                                        ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_char_p]
        vp, sz, cp = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p
        L.orc_sha256.argtypes = [cp, sz, cp]
        L.orc_binius_prove.argtypes = [ctypes.c_uint, cp, sz, sz, cp, sz, vp, sz, vp, cp, sz, ctypes.c_int, cp, cp]
        L.orc_binius_verify.argtypes = [ctypes.c_uint, cp, sz, sz, cp, sz, vp, sz, vp, cp, sz, ctypes.c_int, cp, cp]
        L.orc_binius_fold.argtypes = [ctypes.c_uint, cp, sz, sz, cp, cp]
        L.orc_binius_interpolate.argtypes = [ctypes.c_uint, cp, sz, cp]
        L.orc_binius_challenges.argtypes = [ctypes.c_uint, cp, sz, cp, sz, cp]
        L.orc_circle_twiddles.argtypes = [ctypes.c_uint, u32p]
        L.orc_merkle_root.argtypes = [ctypes.c_char_p, ctypes.c_size_t, u8p]
        L.orc_interpolate_subgroup.argtypes = [u32p, ctypes.c_uint, ctypes.c_int, u32p]
        L.orc_evaluate_coset.argtypes = [u32p, ctypes.c_size_t, ctypes.c_uint, ctypes.c_int, u32p]
        L.orc_channel_script.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                         ctypes.c_size_t, u32p, ctypes.c_size_t, ctypes.c_uint64, u64p]
        L.orc_fri_prove_codeword.argtypes = [ctypes.c_uint8, ctypes.c_uint8, ctypes.c_uint64, ctypes.c_uint8,
                                             u32p, ctypes.c_char_p, ctypes.c_size_t,
                                             ctypes.POINTER(u8p), ctypes.POINTER(ctypes.c_size_t)]
        L.orc_fri_verify.argtypes = [ctypes.c_uint8, ctypes.c_uint8, ctypes.c_uint64, ctypes.c_uint8,
                                     ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                     ctypes.POINTER(ctypes.c_int)]
        L.orc_prove.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int,
                                ctypes.POINTER(u8p), ctypes.POINTER(ctypes.c_size_t)]
        L.orc_verify.argtypes = [ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                 ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                 ctypes.c_size_t, ctypes.POINTER(ctypes.c_int)]
        L.orc_proof_roundtrip.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(u8p),
                                          ctypes.POINTER(ctypes.c_size_t)]
        L.orc_commit_columns.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint, ctypes.c_uint, u8p]
        L.orc_circle_commit.argtypes = [u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, u32p, u32p,
                                        ctypes.c_uint32, ctypes.c_int, ctypes.c_int, u8p, u8p, u32p, u32p, u32p]
        _lib = L
    return _lib


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(u32p)


def _out_u32(shape):
    a = np.zeros(shape, dtype=np.uint32)
    return a, a.ctypes.data_as(u32p)


def _take_bytes(ptr, n):
    data = ctypes.string_at(ptr, n.value)
    lib().orc_free(ptr)
    return data


def blake3(msg: bytes) -> bytes:
    out = (ctypes.c_uint8 * 32)()
    lib().orc_blake3(msg, len(msg), out)
    return bytes(out)


def hash2(a: bytes, b: bytes) -> bytes:
    out = (ctypes.c_uint8 * 32)()
    lib().orc_hash2(a, b, out)
    return bytes(out)


def hash_qm31(v):
    v, p = _u32(v)
    n = v.size // 4
    out = np.zeros((n, 32), dtype=np.uint8)
    lib().orc_hash_qm31(p, n, out.ctypes.data_as(u8p))
    return out


def hash_m31_rows(rows):
    rows, p = _u32(rows)
    out = np.zeros((rows.shape[0], 32), dtype=np.uint8)
    lib().orc_hash_m31_rows(p, rows.shape[0], rows.shape[1], out.ctypes.data_as(u8p))
    return out


_OPS = {"add": 0, "sub": 1, "mul": 2, "neg": 3, "inv": 4}


def m31_op(op, a, b=None):
    a, pa = _u32(a)
    pb = None
    if b is not None:
        b, pb = _u32(b)
    out, po = _out_u32(a.shape)
    lib().orc_m31_op(_OPS[op], pa, pb, po, a.size)
    return out


def qm31_op(op, a, b=None):
    a, pa = _u32(a)
    pb = None
    if b is not None:
        b, pb = _u32(b)
    out, po = _out_u32(a.shape)
    lib().orc_qm31_op(_OPS[op], pa, pb, po, a.size // 4)
    return out


def qm31_pow(a, e):
    a, pa = _u32(a)
    out, po = _out_u32((4,))
    lib().orc_qm31_pow(pa, e, po)
    return out


def qm31_root(log_size):
    out, po = _out_u32((4,))
    lib().orc_qm31_root(log_size, po)
    return out


def circle_generator_mul(scalar):
    out, po = _out_u32((2,))
    lib().orc_circle_generator_mul(scalar, po)
    return tuple(int(x) for x in out)


def circle_domain(log_n):
    xs, px = _out_u32((1 << log_n,))
    ys, py = _out_u32((1 << log_n,))
    lib().orc_circle_domain(log_n, px, py)
    return xs, ys


def circle_fft(coeffs, faithful=False):
    coeffs, p = _u32(coeffs)
    log_n = coeffs.size.bit_length() - 1
    out, po = _out_u32(coeffs.shape)
    lib().orc_circle_fft(p, log_n, po, int(faithful))
    return out


def circle_ifft(evals, faithful=False):
    evals, p = _u32(evals)
    log_n = evals.size.bit_length() - 1
    out, po = _out_u32(evals.shape)
    lib().orc_circle_ifft(p, log_n, po, int(faithful))
    return out


def circle_eval_at(coeffs, x, y):
    coeffs, p = _u32(coeffs)
    return int(lib().orc_circle_eval_at(p, coeffs.size.bit_length() - 1, x, y))


def circle_twiddles(log_n):
    out, po = _out_u32((1 << (log_n - 1),))
    lib().orc_circle_twiddles(log_n, po)
    return out


def merkle_root(leaves):
    leaves = np.ascontiguousarray(leaves, dtype=np.uint8)
    out = (ctypes.c_uint8 * 32)()
    lib().orc_merkle_root(leaves.tobytes(), leaves.shape[0], out)
    return bytes(out)


def interpolate_subgroup(ys, use_ntt=False):
    ys, p = _u32(ys)
    n = ys.size // 4
    out, po = _out_u32((n, 4))
    lib().orc_interpolate_subgroup(p, n.bit_length() - 1, int(use_ntt), po)
    return out


def evaluate_coset(coeffs, log_N, use_ntt=False):
    coeffs, p = _u32(coeffs)
    out, po = _out_u32((1 << log_N, 4))
    lib().orc_evaluate_coset(p, coeffs.size // 4, log_N, int(use_ntt), po)
    return out


def channel_script(sep: bytes, absorb: bytes, n_qm31=0, n_idx=0, idx_bound=1):
    q, pq = _out_u32((max(n_qm31, 1), 4))
    idx = np.zeros(max(n_idx, 1), dtype=np.uint64)
    lib().orc_channel_script(sep, len(sep), absorb, len(absorb), n_qm31, pq, n_idx, idx_bound,
                             idx.ctypes.data_as(u64p))
    return q[:n_qm31], idx[:n_idx]


def fri_prove_codeword(log_size, log_blowup, num_queries, remainder_log, codeword, sep: bytes):
    cw, p = _u32(codeword)
    out = u8p()
    n = ctypes.c_size_t()
    rc = lib().orc_fri_prove_codeword(log_size, log_blowup, num_queries, remainder_log, p, sep, len(sep),
                                      ctypes.byref(out), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"orc_fri_prove_codeword failed: {rc}")
    return _take_bytes(out, n)


def fri_verify(log_size, log_blowup, num_queries, remainder_log, proof: bytes, sep: bytes):
    ok = ctypes.c_int()
    rc = lib().orc_fri_verify(log_size, log_blowup, num_queries, remainder_log, proof, len(proof), sep,
                              len(sep), ctypes.byref(ok))
    if rc != 0:
        return False
    return bool(ok.value)


def prove(air_id, params: bytes, public_inputs: bytes, preprocessed: bytes, trace: bytes, sep: bytes,
          mode=1):
    out = u8p()
    n = ctypes.c_size_t()
    rc = lib().orc_prove(air_id, params, len(params), public_inputs, len(public_inputs), preprocessed,
                         len(preprocessed), trace, len(trace), sep, len(sep), mode, ctypes.byref(out),
                         ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"orc_prove failed: {rc}")
    return _take_bytes(out, n)


def verify(air_id, params: bytes, public_inputs: bytes, proof: bytes, sep: bytes):
    ok = ctypes.c_int()
    rc = lib().orc_verify(air_id, params, len(params), public_inputs, len(public_inputs), proof, len(proof),
                          sep, len(sep), ctypes.byref(ok))
    if rc != 0:
        return False
    return bool(ok.value)


def proof_roundtrip(proof: bytes):
    out = u8p()
    n = ctypes.c_size_t()
    rc = lib().orc_proof_roundtrip(proof, len(proof), ctypes.byref(out), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"orc_proof_roundtrip failed: {rc}")
    return _take_bytes(out, n)


def circle_commit(trace, log_blowup, gammas, alphas, faithful=False, threads=None, keep_lde=False):
    """trace: (n_cols, 2^log_rows) uint32. Returns dict(lde_root, layer_roots, final_layer[, lde, g])."""
    trace, pt = _u32(trace)
    n_cols, n = trace.shape
    log_rows = n.bit_length() - 1
    log_N = log_rows + log_blowup
    gammas, pg = _u32(gammas)
    alphas, pa = _u32(alphas)
    n_folds = alphas.size // 4
    root = (ctypes.c_uint8 * 32)()
    layer_roots = np.zeros((n_folds, 32), dtype=np.uint8)
    final, pf = _out_u32((1 << (log_N - n_folds), 4))
    lde = g = None
    pl = pgo = None
    if keep_lde:
        lde, pl = _out_u32((n_cols, 1 << log_N))
        g, pgo = _out_u32((1 << log_N, 4))
    threads = threads or os.cpu_count() or 1
    rc = lib().orc_circle_commit(pt, n_cols, log_rows, log_blowup, pg, pa, n_folds, int(faithful), threads,
                                 root, layer_roots.ctypes.data_as(u8p), pf, pl, pgo)
    if rc != 0:
        raise RuntimeError(f"orc_circle_commit failed: {rc}")
    res = {"lde_root": bytes(root), "layer_roots": layer_roots, "final_layer": final}
    if keep_lde:
        res["lde"] = lde
        res["g"] = g
    return res


def commit_columns(columns: bytes, n_columns, trace_log, log_blowup):
    out = (ctypes.c_uint8 * (32 * max(n_columns, 1)))()
    rc = lib().orc_commit_columns(columns, len(columns), trace_log, log_blowup, out)
    if rc != 0:
        raise RuntimeError(f"orc_commit_columns failed: {rc}")
    return [bytes(out)[32 * j:32 * j + 32] for j in range(n_columns)]


def tower_mul(level, a, b):
    """Binius tower multiply (src/binius/tower.zig mulRec) of two ints < 2^(2^level)."""
    au = (ctypes.c_uint64 * 2)(a & (2**64 - 1), a >> 64)
    bu = (ctypes.c_uint64 * 2)(b & (2**64 - 1), b >> 64)
    out = (ctypes.c_uint64 * 2)()
    lib().orc_tower_mul(level, au, bu, out)
    return out[0] | (out[1] << 64)


def binius_values(level, cur_flat: bytes, length, m, coeffs: bytes, indices, offsets, dmax, half):
    """One sum-check round's values[t] (src/binius/sumcheck.zig:357-372) in the accelerator
    hook's byte form (level 3: Gf256 bytes, level 7: Gf2_128 16-byte values)."""
    es = 1 if level == 3 else 16
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    off = np.ascontiguousarray(offsets, dtype=np.uint32)
    out = ctypes.create_string_buffer((dmax + 1) * es)
    rc = lib().orc_binius_values(level, cur_flat, length, m, coeffs, len(coeffs) // es, idx.ctypes.data,
                                 idx.size, off.ctypes.data, dmax, half, out)
    if rc != 0:
        raise RuntimeError(f"orc_binius_values failed: {rc}")
    return out.raw


def sha256(msg: bytes) -> bytes:
    """The oracle's SHA-256 (FIPS 180-4), the sum-check transcript hash."""
    out = ctypes.create_string_buffer(32)
    lib().orc_sha256(bytes(msg), len(msg), out)
    return out.raw


def _terms(terms, es):
    """[(indices, coeff int)] -> (coeff bytes, indices array, offsets array)."""
    coeffs = b"".join(int(c).to_bytes(es, "little") for _, c in terms)
    idx = np.array([f for fs, _ in terms for f in fs], dtype=np.uint32)
    off = np.zeros(len(terms) + 1, dtype=np.uint32)
    off[1:] = np.cumsum([len(fs) for fs, _ in terms])
    return coeffs, idx, off


def binius_prove(level, tables: bytes, k, m, terms, seed=None):
    """Sumcheck(F).proveCombination (its optional transcript seed when seed is bytes) over
    TowerField(level), level 3 or 7: tables = m tables of 2^k elements, little-endian.
    Returns (claimed bytes, rounds bytes: k * (dmax + 1) elements)."""
    es = 1 if level == 3 else 16
    coeffs, idx, off = _terms(terms, es)
    dmax = max(len(fs) for fs, _ in terms)
    claimed = ctypes.create_string_buffer(es)
    rounds = ctypes.create_string_buffer(max(1, k * (dmax + 1) * es))
    sd = b"" if seed is None else bytes(seed)
    rc = lib().orc_binius_prove(level, bytes(tables), k, m, coeffs, len(terms), idx.ctypes.data, idx.size,
                                off.ctypes.data, sd, len(sd), int(seed is not None), claimed, rounds)
    if rc != 0:
        raise RuntimeError(f"orc_binius_prove failed: {rc}")
    return claimed.raw, rounds.raw[:k * (dmax + 1) * es]


def binius_verify(level, tables: bytes, k, m, terms, claimed: bytes, rounds: bytes, seed=None):
    """True when the proof's rounds replay and end at g(challenges) (sumcheck.zig:632-665)."""
    es = 1 if level == 3 else 16
    coeffs, idx, off = _terms(terms, es)
    sd = b"" if seed is None else bytes(seed)
    rc = lib().orc_binius_verify(level, bytes(tables), k, m, coeffs, len(terms), idx.ctypes.data, idx.size,
                                 off.ctypes.data, sd, len(sd), int(seed is not None), bytes(claimed),
                                 bytes(rounds) or b"\0")
    if rc < 0:
        raise RuntimeError(f"orc_binius_verify failed: {rc}")
    return rc == 1


def binius_fold(level, tables: bytes, length, m, r: int):
    """m tables of `length` elements folded at r into m tables of length // 2."""
    es = 1 if level == 3 else 16
    out = ctypes.create_string_buffer(max(1, m * (length // 2) * es))
    rc = lib().orc_binius_fold(level, bytes(tables), length, m, int(r).to_bytes(es, "little"), out)
    if rc != 0:
        raise RuntimeError(f"orc_binius_fold failed: {rc}")
    return out.raw[:m * (length // 2) * es]


def binius_interpolate(level, values):
    """Low-first coefficients of the polynomial through (t, values[t]), t = 0..n-1."""
    es = 1 if level == 3 else 16
    out = ctypes.create_string_buffer(len(values) * es)
    rc = lib().orc_binius_interpolate(level, b"".join(int(v).to_bytes(es, "little") for v in values),
                                      len(values), out)
    if rc != 0:
        raise RuntimeError(f"orc_binius_interpolate failed: {rc}")
    return [int.from_bytes(out.raw[i * es:(i + 1) * es], "little") for i in range(len(values))]


def binius_challenges(level, seed: bytes, elems):
    """Transcript.initBytes(seed), then absorb([e]) for each e: the challenges."""
    es = 1 if level == 3 else 16
    out = ctypes.create_string_buffer(max(1, len(elems) * es))
    rc = lib().orc_binius_challenges(level, bytes(seed), len(seed),
                                     b"".join(int(e).to_bytes(es, "little") for e in elems) or b"\0",
                                     len(elems), out)
    if rc != 0:
        raise RuntimeError(f"orc_binius_challenges failed: {rc}")
    return [int.from_bytes(out.raw[i * es:(i + 1) * es], "little") for i in range(len(elems))]
