"""The Binius sum-check on the GPU (libzs_b200: zs_binius_*) against the oracle
(oracle/binius.hpp, pinned by tests/test_oracle_binius.py) and, where oracle/_ref was
built, against the reference's own GPU kernels (src/cuda/kernels/sumcheck.cu driven as
src/cuda/sumcheck_gpu.zig drives them).

Covered: the values hook over GF(2^8) and GF(2^128) at the shapes of
src/cuda/sumcheck_test.zig (three tables, terms t0 t1 t2 + 2 t0, k = 4..9 and 4..7) and
beyond (2^20 rows, every point count 1..14 on both the register and the looped paths,
empty terms, repeated factors, 256 terms and 1024 factors, half < len / 2, odd len,
half = 0); the device-resident round and fold; the combination prover bit-exact with the
oracle's proveCombination (plain and seeded transcripts, k = 0..10) and, at 2^20 rows,
verified by the oracle's verifier."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TERMS_REF = [([0, 1, 2], 1), ([0], 2)]  # src/cuda/sumcheck_test.zig:40-43


def _flat_terms(terms, es):
    coeffs = b"".join(int(c).to_bytes(es, "little") for _, c in terms)
    idx = [f for fs, _ in terms for f in fs]
    off = [0]
    for fs, _ in terms:
        off.append(off[-1] + len(fs))
    return coeffs, idx, off


def _hook(es):
    from zs_b200 import native
    return native.binius_gf256_values if es == 1 else native.binius_gf128_values


_T8 = None


def _gf256_table(orc):
    """The 64 KB GF(2^8) product table from the oracle's multiply (test-side numpy path)."""
    global _T8
    if _T8 is None:
        _T8 = np.array([orc.tower_mul(3, a, b) for a in range(256) for b in range(256)], dtype=np.uint8)
    return _T8


def _np_values8(orc, cur, length, m, terms, dmax, half):
    """sumcheck.zig:357-372 over GF(2^8), vectorised over the rows with numpy."""
    T = _gf256_table(orc).astype(np.int64)
    tab = np.frombuffer(cur, dtype=np.uint8).reshape(m, length).astype(np.int64)
    out = bytearray()
    for t in range(dmax + 1):
        s = np.zeros(half, dtype=np.int64)
        for fs, c in terms:
            prod = np.full(half, c, dtype=np.int64)
            for f in fs:
                a, b = tab[f, 0:2 * half:2], tab[f, 1:2 * half:2]
                prod = T[prod * 256 + (a ^ T[t * 256 + (a ^ b)])]
            s ^= prod
        out.append(int(np.bitwise_xor.reduce(s)) if half else 0)
    return bytes(out)


@pytest.mark.parametrize("level,k", [(3, 1), (3, 4), (3, 6), (3, 9), (3, 12), (7, 1), (7, 4), (7, 5), (7, 7),
                                     (7, 9)])
def test_hook_reference_shapes_match_oracle(orc, level, k):
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(700 + 10 * level + k)
    n = 1 << k
    cur = rng.bytes(3 * n * es)
    coeffs, idx, off = _flat_terms(TERMS_REF, es)
    got = _hook(es)(cur, n, 3, coeffs, idx, off, 3, n // 2)
    assert got == orc.binius_values(level, cur, n, 3, coeffs, idx, off, 3, n // 2)


@pytest.mark.parametrize("dmax", list(range(0, 14)))
@pytest.mark.parametrize("level", [3, 7])
def test_hook_every_point_count(orc, level, dmax):
    """dmax + 1 <= 8 points run in registers, more in one pass per point; terms of every
    length 0..dmax with repeated factors."""
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(900 + 20 * level + dmax)
    m, n = 4, 64 if level == 7 else 512
    cur = rng.bytes(m * n * es)
    terms = [([(3 * j + i) % m for j in range(d)], int(rng.integers(1, 256))) for i, d in
             enumerate(sorted({0, dmax, max(dmax - 1, 0), dmax // 2}))]
    coeffs, idx, off = _flat_terms(terms, es)
    got = _hook(es)(cur, n, m, coeffs, idx, off, dmax, n // 2)
    assert got == orc.binius_values(level, cur, n, m, coeffs, idx, off, dmax, n // 2)


@pytest.mark.parametrize("level", [3, 7])
@pytest.mark.parametrize("shape", ["short_half", "odd_len", "zero_half", "one_row_pair", "max_terms"])
def test_hook_edge_shapes(orc, level, shape):
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(zlib.crc32(f"{level}:{shape}".encode()))
    m, length, half, terms = 3, 256, 128, TERMS_REF
    if shape == "short_half":
        half = 125
    elif shape == "odd_len":
        length, half = 257, 128
    elif shape == "zero_half":
        half = 0
    elif shape == "one_row_pair":
        length, half = 2, 1
    elif shape == "max_terms":  # 256 terms, 1024 factor indices over 7 tables
        m, length, half = 7, 32 if level == 3 else 16, 16 if level == 3 else 8
        terms = [([(k + j) % m for j in range(4)], (k * 37 + 1) & 0xff) for k in range(256)]
    cur = rng.bytes(m * length * es)
    dmax = max(len(fs) for fs, _ in terms)
    coeffs, idx, off = _flat_terms(terms, es)
    got = _hook(es)(cur, length, m, coeffs, idx, off, dmax, half)
    assert got == orc.binius_values(level, cur, length, m, coeffs, idx, off, dmax, half)
    if shape == "zero_half":
        assert got == bytes((dmax + 1) * es)


@pytest.mark.parametrize("k", [16, 20])
def test_hook_gf256_full_size(orc, k):
    """2^20 rows against a numpy evaluation over the oracle's product table, and the
    hypercube sum values[0] + values[1] against the direct combination sum."""
    rng = np.random.default_rng(k)
    n = 1 << k
    cur = rng.bytes(3 * n)
    coeffs, idx, off = _flat_terms(TERMS_REF, 1)
    got = _hook(1)(cur, n, 3, coeffs, idx, off, 3, n // 2)
    assert got == _np_values8(orc, cur, n, 3, TERMS_REF, 3, n // 2)
    T = _gf256_table(orc).astype(np.int64)
    t0, t1, t2 = (np.frombuffer(cur, dtype=np.uint8).reshape(3, n).astype(np.int64))
    direct = np.bitwise_xor.reduce(T[T[t0 * 256 + t1] * 256 + t2] ^ T[2 * 256 + t0])
    assert got[0] ^ got[1] == int(direct)


def _dev(buf: bytes):
    import torch
    return torch.frombuffer(bytearray(buf), dtype=torch.uint8).to("cuda")


@pytest.mark.parametrize("level", [3, 7])
def test_device_round_and_fold_match_oracle(orc, level):
    """zs_binius_sumcheck_values_device and zs_binius_sumcheck_fold_device on tables in
    device memory: the round's values, then the fold at a random r, then the next round
    on the folded tables."""
    import torch
    from zs_b200 import native
    es = 1 if level == 3 else 16
    bits = 8 if level == 3 else 128
    rng = np.random.default_rng(1234 + level)
    m, n = 3, 1024 if level == 3 else 256
    cur = rng.bytes(m * n * es)
    d_cur = _dev(cur)
    d_out = torch.zeros(4 * 4 * 4, dtype=torch.uint8, device="cuda")
    d_next = torch.zeros(m * (n // 2) * es, dtype=torch.uint8, device="cuda")
    d_scratch = torch.zeros(65536, dtype=torch.uint8, device="cuda")
    coeffs, idx, off = _flat_terms(TERMS_REF, es)
    native.binius_values_device(bits, d_cur.data_ptr(), n, m, TERMS_REF, 3, n // 2, d_out.data_ptr())
    torch.cuda.synchronize()
    assert bytes(d_out.cpu().numpy())[:4 * es] == orc.binius_values(level, cur, n, m, coeffs, idx, off, 3, n // 2)
    r = int.from_bytes(rng.bytes(es), "little")
    native.binius_fold_device(bits, d_cur.data_ptr(), n, m, r, d_next.data_ptr(), d_scratch.data_ptr())
    torch.cuda.synchronize()
    folded = orc.binius_fold(level, cur, n, m, r)
    assert bytes(d_next.cpu().numpy()) == folded
    native.binius_values_device(bits, d_next.data_ptr(), n // 2, m, TERMS_REF, 3, n // 4, d_out.data_ptr())
    torch.cuda.synchronize()
    assert bytes(d_out.cpu().numpy())[:4 * es] == orc.binius_values(level, folded, n // 2, m, coeffs, idx, off, 3,
                                                                      n // 4)


@pytest.mark.parametrize("level,k,seed", [(3, 0, None), (3, 1, None), (3, 2, b"root"), (3, 5, None), (3, 10, None),
                                          (3, 10, b"\x07" * 32), (7, 0, None), (7, 1, None), (7, 3, b"seed"),
                                          (7, 6, None)])
def test_prover_matches_oracle(orc, level, k, seed):
    """zs_binius_sumcheck_prove_combination against the oracle's proveCombination:
    the claimed sum and every round's coefficients, byte for byte."""
    from zs_b200 import native
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(50 + 11 * k + level)
    tables = rng.bytes(3 * (1 << k) * es)
    got = native.binius_prove_combination(8 if level == 3 else 128, tables, k, 3, TERMS_REF, seed)
    assert got == orc.binius_prove(level, tables, k, 3, TERMS_REF, seed)


@pytest.mark.parametrize("level", [3, 7])
def test_prover_mixed_terms_matches_oracle(orc, level):
    """The combination test of sumcheck.zig:632-665 (2 t0 t2 + 3 t1) and a wider one
    (five tables, degree 6, repeated factors)."""
    from zs_b200 import native
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(77 + level)
    for m, terms, k in ((3, [([0, 2], 2), ([1], 3)], 4),
                        (5, [([0, 1, 2, 3, 4, 0], 9), ([4, 4], 1), ([], 7), ([2], 200)], 6 if level == 3 else 3)):
        tables = rng.bytes(m * (1 << k) * es)
        got = native.binius_prove_combination(8 if level == 3 else 128, tables, k, m, terms)
        assert got == orc.binius_prove(level, tables, k, m, terms)
        assert orc.binius_verify(level, tables, k, m, terms, *got)


@pytest.mark.parametrize("level,k", [(3, 20), (7, 13)])
def test_prover_full_size_verifies(orc, level, k):
    """At 2^20 rows (GF(2^8)) and 2^13 (GF(2^128)): the oracle's verifier accepts the
    device proof (rounds replay, final sum = g at the challenges), and rejects it with
    one coefficient changed."""
    from zs_b200 import native
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(k)
    tables = rng.bytes(3 * (1 << k) * es)
    claimed, rounds = native.binius_prove_combination(8 if level == 3 else 128, tables, k, 3, TERMS_REF)
    assert orc.binius_verify(level, tables, k, 3, TERMS_REF, claimed, rounds)
    bad = bytearray(rounds)
    bad[len(bad) // 2] ^= 0x5a
    assert not orc.binius_verify(level, tables, k, 3, TERMS_REF, claimed, bytes(bad))


def _ref():
    import ref_gpu
    if not ref_gpu.sumcheck_available():
        pytest.skip("oracle/_ref not built: the reference tree was absent when build() ran")
    return ref_gpu


@pytest.mark.parametrize("level,k", [(3, 4), (3, 6), (3, 9), (3, 20), (7, 4), (7, 7), (7, 16)])
def test_reference_gpu_kernel_agrees(orc, level, k):
    """The reference's own kernels at the shapes src/cuda/sumcheck_test.zig benchmarks
    (and 2^20 / 2^16 rows): the same values as this library's hook."""
    ref = _ref()
    es = 1 if level == 3 else 16
    rng = np.random.default_rng(3000 + 10 * level + k)
    n = 1 << k
    cur = rng.bytes(3 * n * es)
    coeffs, idx, off = _flat_terms(TERMS_REF, es)
    want, _, _ = ref.sumcheck_values(level == 7, cur, n, 3, coeffs, idx, off, 3, n // 2)
    assert _hook(es)(cur, n, 3, coeffs, idx, off, 3, n // 2) == want
    if k <= 9:
        assert want == orc.binius_values(level, cur, n, 3, coeffs, idx, off, 3, n // 2)
