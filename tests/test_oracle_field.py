"""Oracle field tower against the reference's known answers and a big-int model.

Restates the inline tests of src/m31/field/{m31,cm31,qm31}.zig.
"""
import numpy as np

from zs_b200 import workload as wl

P = 2**31 - 1
rng = np.random.default_rng(42)


def test_m31_against_u64(orc):
    # m31.zig:159-173
    a = rng.integers(0, P, 1000, dtype=np.uint64)
    b = rng.integers(0, P, 1000, dtype=np.uint64)
    assert np.array_equal(orc.m31_op("add", a, b), (a + b) % P)
    assert np.array_equal(orc.m31_op("sub", a, b), (a + P - b) % P)
    assert np.array_equal(orc.m31_op("mul", a, b), (a * b) % P)


def test_m31_edge_cases(orc):
    # m31.zig:174-189
    mx = P - 1
    pairs = [(0, 0, "add", 0), (0, 1, "add", 1), (mx, 1, "add", 0), (1, mx, "add", 0),
             (mx, mx, "sub", 0), (0, 1, "sub", mx), (mx, mx, "mul", 1), (0, mx, "mul", 0)]
    for x, y, op, want in pairs:
        assert orc.m31_op(op, [x], [y])[0] == want
    assert orc.m31_op("neg", [1])[0] == mx
    assert orc.m31_op("neg", [0])[0] == 0


def test_m31_inverse_and_fermat(orc):
    # m31.zig:198-224
    a = rng.integers(1, P, 200, dtype=np.uint64)
    inv = orc.m31_op("inv", a)
    assert np.all(orc.m31_op("mul", a, inv) == 1)
    assert orc.m31_op("inv", [1])[0] == 1
    # inv(0) is 0^(p-2) = 0 in release builds of the reference.
    assert orc.m31_op("inv", [0])[0] == 0


def _cm(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def test_qm31_against_bigint_model(orc):
    # qm31.zig:150-168 (reference refQMMul) with an independent Python model
    a = rng.integers(0, P, (300, 4), dtype=np.uint64)
    b = rng.integers(0, P, (300, 4), dtype=np.uint64)
    got = orc.qm31_op("mul", a, b)
    for i in range(300):
        want = wl.qm_mul(tuple(int(x) for x in a[i]), tuple(int(x) for x in b[i]))
        assert tuple(int(x) for x in got[i]) == want
    assert np.array_equal(orc.qm31_op("add", a, b), (a + b) % P)
    assert np.array_equal(orc.qm31_op("sub", a, b), (a + P - b) % P)


def test_qm31_tower_identity(orc):
    # qm31.zig:170-180: j^2 = -i
    j = np.array([[0, 0, 1, 0]], dtype=np.uint32)
    assert orc.qm31_op("mul", j, j).tolist() == [[0, P - 1, 0, 0]]
    i = np.array([[0, 1, 0, 0]], dtype=np.uint32)
    assert orc.qm31_op("mul", i, i).tolist() == [[P - 1, 0, 0, 0]]


def test_qm31_inverse(orc):
    # qm31.zig:182-193
    a = rng.integers(0, P, (100, 4), dtype=np.uint64)
    inv = orc.qm31_op("inv", a)
    prod = orc.qm31_op("mul", a, inv)
    assert np.all(prod == np.array([1, 0, 0, 0]))


def test_qm31_two_adic_root(orc):
    # qm31.zig:80-83 bytes, qm31.zig:195-209 order 2^32 and primitive roots
    root = orc.qm31_root(32)
    raw = bytes([0x60, 0x1f, 0x3d, 0x34, 0x32, 0x39, 0xa0, 0x6a, 0xa0, 0xd6, 0x51, 0x61, 0x91, 0xe7, 0x86, 0x3e])
    assert root.astype("<u4").tobytes() == raw
    assert orc.qm31_pow(root, 1 << 32).tolist() == [1, 0, 0, 0]
    assert orc.qm31_pow(root, 1 << 31).tolist() == [P - 1, 0, 0, 0]
    for log in range(0, 13):
        w = orc.qm31_root(log)
        assert orc.qm31_pow(w, 1 << log).tolist() == [1, 0, 0, 0]
        if log > 0:
            assert orc.qm31_pow(w, 1 << (log - 1)).tolist() != [1, 0, 0, 0]


def test_byte_encodings():
    # m31.zig:258-262, cm31.zig:154-157, qm31.zig:222-225
    from zs_b200 import wire
    assert wire.qm31((1, 0, 0, 0))[0] == 1 and wire.qm31((1, 0, 0, 0))[15] == 0
    enc_i = wire.qm31((0, 1, 0, 0))
    assert enc_i[0] == 0 and enc_i[4] == 1
