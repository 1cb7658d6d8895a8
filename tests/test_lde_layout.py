"""Index maps of the circle LDE's register-direct passes (k_low10 and the middle pass's
compile-time layout in zig-stark_b200/csrc/circle.cu), restated in Python and checked for
the properties the kernels rely on: every (group, element) of a batch is held by exactly
one thread in each layout, the shared-memory transpose puts each warp's 32 lanes on 32
distinct banks in both layouts, and the global offsets of every launch stay inside the
column and cover it once. No GPU."""
import numpy as np
import pytest

GS = 1060            # words between groups in shared memory (kGS10)
THREADS = 256


def padx(e):
    return e + (e >> 5)


def bitrev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def layouts():
    tid = np.arange(THREADS)
    strided = (tid >> 5, tid & 31)      # group, r: elements r + 32 m
    consecutive = (tid & 7, tid >> 3)   # group, r: elements 32 r + m
    return strided, consecutive


def test_each_layout_holds_every_element_once():
    (gs, rs), (gc, rc) = layouts()
    a = {(int(g), int(r) + 32 * m) for g, r in zip(gs, rs) for m in range(32)}
    b = {(int(g), 32 * int(r) + m) for g, r in zip(gc, rc) for m in range(32)}
    assert len(a) == len(b) == 8 * 1024


def test_shared_offsets_are_padded_group_offsets_and_bank_conflict_free():
    (gs, rs), (gc, rc) = layouts()
    assert GS % 32 == 4 and GS >= padx(1023) + 1
    assert 2 * 8 * GS * 4 <= 227 * 1024
    for m in range(32):
        # strided_at(s, g, r)[33 m] and consecutive_at(s, g, r)[m]
        so = gs * GS + rs + 33 * m
        co = gc * GS + 33 * rc + m
        assert np.array_equal(so, gs * GS + np.array([padx(int(r) + 32 * m) for r in rs]))
        assert np.array_equal(co, gc * GS + np.array([padx(32 * int(r) + m) for r in rc]))
        for w in range(8):
            assert len(set((so[32 * w:32 * w + 32] % 32).tolist())) == 32
            assert len(set((co[32 * w:32 * w + 32] % 32).tolist())) == 32


@pytest.mark.parametrize("LG", [13, 16, 20])
def test_low_pass_global_offsets_cover_the_column_once(LG):
    (gs, rs), (gc, rc) = layouts()
    hb, N = LG - 10, 1 << LG
    rev = np.zeros(N, np.int64)
    con = np.zeros(N, np.int64)
    for g0 in range(0, 1 << hb, 8):
        for g, r in zip(gc, rc):
            base = (bitrev(int(r), 5) << hb) + g0 + int(g)
            for m in range(32):
                idx = base + (bitrev(m, 5) << (hb + 5))
                # element 32 r + m of group g0 + g in the bit-reversed order
                assert idx == (bitrev(32 * int(r) + m, 10) << hb) + g0 + int(g)
                rev[idx] += 1
        for g, r in zip(gs, rs):
            vs = bitrev(g0 + int(g), hb)
            for m in range(32):
                con[(vs << 10) + int(r) + 32 * m] += 1
    assert (rev == 1).all() and (con == 1).all()


def test_middle_pass_global_offsets_cover_the_column_once():
    (_, _), (gc, rc) = layouts()
    n = 1 << 20
    seen = np.zeros(n, np.int64)
    for lo0 in range(0, 1024, 8):
        io = (rc.astype(np.int64) << 15) + lo0 + gc
        for m in range(32):
            seen[io + (m << 10)] += 1
    assert (seen == 1).all()
