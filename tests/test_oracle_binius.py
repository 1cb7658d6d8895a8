"""The oracle's Binius tower field and sum-check round against the reference's own tests
(src/binius/tower.zig:377-470, src/binius/sumcheck.zig:571-600): GF(4) at level 1, the
defining polynomial y^2 + beta y + 1 = 0 at every level, field axioms on random
elements at every level, exhaustive checks of GF(16) and GF(256) (every nonzero
element invertible: its powers cycle back to 1), and a sum-check round's values[t]
against a direct Python evaluation built on the oracle's multiply."""
import numpy as np
import pytest

MASK64 = 2**64 - 1


def _rng(level, seed):
    # tower.zig:372-375: an LCG, fromInt keeps the low 2^level bits
    bits = 1 << level
    while True:
        seed = (seed * 6364136223846793005 + 1442695040888963407) & MASK64
        yield seed & ((1 << bits) - 1) if bits < 128 else seed


def test_level1_is_gf4(orc):
    x0 = 0b10  # alpha at level 1
    assert orc.tower_mul(1, x0, x0) == x0 ^ 1  # X_0^2 = X_0 + 1
    assert orc.tower_mul(1, orc.tower_mul(1, x0, x0), x0) == 1


@pytest.mark.parametrize("level", range(1, 8))
def test_field_polynomial_every_level(orc, level):
    y = 1 << (1 << (level - 1))  # alpha: the root X_(level-1)
    beta = 1 if level == 1 else 1 << (1 << (level - 2))
    assert orc.tower_mul(level, y, y) ^ orc.tower_mul(level, beta, y) ^ 1 == 0


@pytest.mark.parametrize("level", range(1, 8))
def test_field_axioms_random(orc, level):
    g = _rng(level, level)
    for _ in range(100):
        a, b, c = next(g), next(g), next(g)
        m = lambda x, y: orc.tower_mul(level, x, y)  # noqa: E731
        assert m(a, b ^ c) == m(a, b) ^ m(a, c)
        assert m(m(a, b), c) == m(a, m(b, c))
        assert m(a, b) == m(b, a)
        assert m(a, 1) == a


@pytest.mark.parametrize("level", [2, 3])
def test_small_fields_exhaustive(orc, level):
    n = 1 << (1 << level)
    table = [[orc.tower_mul(level, a, b) for b in range(n)] for a in range(n)]
    for a in range(1, n):
        assert sorted(table[a][1:]) == list(range(1, n))  # a * (.) permutes the nonzero elements
        assert any(table[a][b] == 1 for b in range(1, n))


@pytest.mark.parametrize("level,dmax", [(3, 3), (7, 3), (3, 5), (7, 1)])
def test_round_values_against_direct_evaluation(orc, level, dmax):
    """sumcheck.zig:357-372 evaluated directly in Python with the oracle's multiply."""
    rng = np.random.default_rng(level * 10 + dmax)
    es = 1 if level == 3 else 16
    m, half = 3, 8
    length = 2 * half
    vals = [[int.from_bytes(rng.bytes(es), "little") for _ in range(length)] for _ in range(m)]
    terms = [([0, 1, 2], 1), ([0], 2)] if dmax == 3 else ([([0, 1, 2, 0, 1], 7), ([2], 3)] if dmax == 5
                                                          else [([1], 5), ([2], 9)])
    indices = [f for fs, _ in terms for f in fs]
    offsets = [0]
    for fs, _ in terms:
        offsets.append(offsets[-1] + len(fs))
    cur_flat = b"".join(v.to_bytes(es, "little") for col in vals for v in col)
    coeffs = b"".join(c.to_bytes(es, "little") for _, c in terms)
    got = orc.binius_values(level, cur_flat, length, m, coeffs, indices, offsets, dmax, half)
    mul = lambda x, y: orc.tower_mul(level, x, y)  # noqa: E731
    for t in range(dmax + 1):
        s = 0
        for rest in range(half):
            for fs, c in terms:
                prod = c
                for f in fs:
                    a, b = vals[f][2 * rest], vals[f][2 * rest + 1]
                    prod = mul(prod, a ^ mul(t, a ^ b))
                s ^= prod
        assert int.from_bytes(got[t * es:(t + 1) * es], "little") == s


# ---- the transcript, interpolation and the combination prover ------------------------

@pytest.mark.parametrize("n", [0, 1, 3, 55, 56, 63, 64, 65, 119, 1000])
def test_sha256_matches_hashlib(orc, n):
    import hashlib
    msg = bytes((7 * i + 3) & 0xff for i in range(n))
    assert orc.sha256(msg) == hashlib.sha256(msg).digest()


@pytest.mark.parametrize("level,n", [(3, 1), (3, 2), (3, 4), (3, 9), (7, 2), (7, 4), (7, 6)])
def test_interpolation_recovers_polynomial(orc, level, n):
    """sumcheck.zig:576-605 (recover a linear and a quadratic polynomial), over the
    hook's fields and more points: values at t = 0..n-1 of known coefficients give the
    coefficients back."""
    g = _rng(level, 100 + n)
    coeffs = [next(g) for _ in range(n)]
    mul = lambda x, y: orc.tower_mul(level, x, y)  # noqa: E731
    values = []
    for t in range(n):
        acc = 0
        for c in reversed(coeffs):
            acc = mul(acc, t) ^ c
        values.append(acc)
    assert orc.binius_interpolate(level, values) == coeffs


def _py_prove(orc, level, k, tables, terms, seed=None):
    """proveCombination (sumcheck.zig:232-395) in Python over the oracle's multiply and
    hashlib's SHA-256: an independent restatement for small cases."""
    import hashlib
    es = 1 if level == 3 else 16
    mul = lambda x, y: orc.tower_mul(level, x, y)  # noqa: E731
    n = 1 << k
    dmax = max(len(fs) for fs, _ in terms)
    h = 0
    for x in range(n):
        for fs, c in terms:
            p = c
            for f in fs:
                p = mul(p, tables[f][x])
            h ^= p
    buf = hashlib.sha256(seed if seed is not None else h.to_bytes(es, "little")).digest()
    cur = [list(t) for t in tables]
    rounds = []
    length = n
    for _ in range(k):
        half = length // 2
        values = []
        for t in range(dmax + 1):
            s = 0
            for rest in range(half):
                for fs, c in terms:
                    p = c
                    for f in fs:
                        a, b = cur[f][2 * rest], cur[f][2 * rest + 1]
                        p = mul(p, a ^ mul(t, a ^ b))
                    s ^= p
            values.append(s)
        cs = orc.binius_interpolate(level, values)
        rounds.append(cs)
        buf = hashlib.sha256(buf + b"".join(c.to_bytes(es, "little") for c in cs)).digest()
        r = buf[31] if es == 1 else int.from_bytes(buf[16:], "little")
        for ct in cur:
            for rest in range(half):
                a, b = ct[2 * rest], ct[2 * rest + 1]
                ct[rest] = a ^ mul(r, a ^ b)
        length = half
    return h, rounds


def _flat(tables, es):
    return b"".join(v.to_bytes(es, "little") for t in tables for v in t)


TERMS_REF = [([0, 1, 2], 1), ([0], 2)]  # src/cuda/sumcheck_test.zig:40-43


@pytest.mark.parametrize("level,k,seed", [(3, 1, None), (3, 3, None), (3, 4, b"root"), (7, 2, None),
                                          (7, 3, b"\x00" * 32)])
def test_prover_matches_python_restatement(orc, level, k, seed):
    es = 1 if level == 3 else 16
    g = _rng(level, 7 * k + level)
    tables = [[next(g) for _ in range(1 << k)] for _ in range(3)]
    claimed, rounds = orc.binius_prove(level, _flat(tables, es), k, 3, TERMS_REF, seed)
    h, py_rounds = _py_prove(orc, level, k, tables, TERMS_REF, seed)
    assert int.from_bytes(claimed, "little") == h
    flat = b"".join(c.to_bytes(es, "little") for cs in py_rounds for c in cs)
    assert rounds == flat


@pytest.mark.parametrize("level,k", [(3, 0), (3, 1), (3, 2), (3, 8), (7, 1), (7, 4)])
def test_prove_verify_round_trip_and_tampering(orc, level, k):
    """sumcheck.zig:607-665: the round trip, the claimed sum against the direct
    hypercube combination, and a tampered claim or round that fails."""
    es = 1 if level == 3 else 16
    g = _rng(level, 31 + k)
    # g(x) = 2 t0(x) t2(x) + 3 t1(x), the reference's combination test
    terms = [([0, 2], 2), ([1], 3)]
    tables = [[next(g) for _ in range(1 << k)] for _ in range(3)]
    flat = _flat(tables, es)
    claimed, rounds = orc.binius_prove(level, flat, k, 3, terms)
    assert orc.binius_verify(level, flat, k, 3, terms, claimed, rounds)
    mul = lambda x, y: orc.tower_mul(level, x, y)  # noqa: E731
    direct = 0
    for i in range(1 << k):
        direct ^= mul(2, mul(tables[0][i], tables[2][i])) ^ mul(3, tables[1][i])
    assert int.from_bytes(claimed, "little") == direct
    bad = (int.from_bytes(claimed, "little") ^ 1).to_bytes(es, "little")
    assert not orc.binius_verify(level, flat, k, 3, terms, bad, rounds)
    if k:
        tampered = bytearray(rounds)
        tampered[es] ^= 1
        assert not orc.binius_verify(level, flat, k, 3, terms, claimed, bytes(tampered))


def test_challenges_span_gf256(orc):
    """sumcheck.zig:697-713: 64 absorbs from the seed "challenge-space" reach more than
    16 distinct GF(256) challenges."""
    ch = orc.binius_challenges(3, b"challenge-space", list(range(64)))
    assert len(set(ch)) > 16
