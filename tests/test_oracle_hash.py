"""Oracle Blake3, digests, Merkle trees and channel.

Pins: Blake3("") (src/core/hash/hash.zig:32-43); cross-checks against the `blake3`
package (official BLAKE3 bindings) at every input length the path uses, including the
multi-chunk transcript; an independent Python restatement of the channel
(src/core/channel/channel.zig) built on that package.
"""
import struct

import blake3
import numpy as np
import pytest

rng = np.random.default_rng(7)

EMPTY = bytes.fromhex("af1349b9f5f9a1a6a0404dea36dcc9499bcb25c9adc112b7cc9a93cae41f3262")


def test_blake3_empty_kat(orc):
    assert orc.blake3(b"") == EMPTY


@pytest.mark.parametrize("n", [0, 1, 4, 16, 31, 32, 63, 64, 65, 78, 128, 255, 256, 257, 511, 1023, 1024, 1025,
                               2047, 2048, 2049, 3072, 4096, 5000, 8192, 8193, 16384, 20000, 65537])
def test_blake3_matches_package(orc, n):
    msg = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
    assert orc.blake3(msg) == blake3.blake3(msg).digest()


def test_hash2(orc):
    a = blake3.blake3(b"a").digest()
    b = blake3.blake3(b"b").digest()
    h = orc.hash2(a, b)
    assert h == blake3.blake3(b"zig-stark:pair" + a + b).digest()
    assert h != blake3.blake3(a + b).digest()  # hash.zig:45-53


def test_hash_qm31_and_rows(orc):
    v = rng.integers(0, 2**31 - 1, (50, 4), dtype=np.uint32)
    d = orc.hash_qm31(v)
    for i in range(50):
        assert d[i].tobytes() == blake3.blake3(v[i].astype("<u4").tobytes()).digest()
    rows = rng.integers(0, 2**31 - 1, (20, 64), dtype=np.uint32)
    d = orc.hash_m31_rows(rows)
    for i in range(20):
        assert d[i].tobytes() == blake3.blake3(rows[i].astype("<u4").tobytes()).digest()


def py_merkle_root(leaves):
    level = [bytes(x) for x in leaves]
    while len(level) > 1:
        level = [blake3.blake3(b"zig-stark:pair" + level[2 * i] + level[2 * i + 1]).digest()
                 for i in range(len(level) // 2)]
    return level[0]


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 1024])
def test_merkle_root(orc, n):
    leaves = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    assert orc.merkle_root(leaves) == py_merkle_root(leaves)


def test_merkle_single_leaf(orc):
    # merkle.zig:147-157: root = the leaf
    leaf = blake3.blake3(b"solo").digest()
    assert orc.merkle_root(np.frombuffer(leaf, dtype=np.uint8).reshape(1, 32)) == leaf


class PyChannel:
    """Independent restatement of src/core/channel/channel.zig on the blake3 package."""

    def __init__(self, sep: bytes):
        self.h = blake3.blake3(b"zig-stark:channel" + sep)

    def absorb(self, data: bytes):
        self.h.update(data)

    def sample_bytes(self, n):
        out = b""
        k = 0
        while len(out) < n:
            snap = self.h.copy()
            snap.update(b"zig-stark:sample" + struct.pack("<Q", k))
            blk = snap.digest()
            self.h.update(blk)
            out += blk[: n - len(out)]
            k += 1
        return out

    def sample_qm31(self):
        w = struct.unpack("<4I", self.sample_bytes(16))
        return tuple(x % (2**31 - 1) for x in w)

    def sample_index(self, n):
        bits = n.bit_length()
        nb = (bits + 7) // 8
        mask = (1 << bits) - 1
        while True:
            v = int.from_bytes(self.sample_bytes(nb), "big") & mask
            if v < n:
                return v


@pytest.mark.parametrize("absorb_len", [0, 5, 32, 1000, 3000, 9000])
def test_channel_matches_restatement(orc, absorb_len):
    sep = b"zig-stark:fibonacci:example"
    data = rng.integers(0, 256, absorb_len, dtype=np.uint8).tobytes()
    q, idx = orc.channel_script(sep, data, n_qm31=7, n_idx=40, idx_bound=1 << 14)
    ch = PyChannel(sep)
    ch.absorb(data)
    for i in range(7):
        assert tuple(int(x) for x in q[i]) == ch.sample_qm31()
    for i in range(40):
        assert int(idx[i]) == ch.sample_index(1 << 14)


def test_channel_sample_index_range_and_uniformity(orc):
    # channel.zig:130-157
    for n in (1, 2, 3, 7, 8, 100, 1024):
        _, idx = orc.channel_script(b"idx", b"", n_idx=50, idx_bound=n)
        assert np.all(idx < n)
    _, idx = orc.channel_script(b"uniform", b"", n_idx=4000, idx_bound=8)
    counts = np.bincount(idx.astype(np.int64), minlength=8)
    assert np.all((counts > 200) & (counts < 800))


def test_channel_determinism(orc):
    a, _ = orc.channel_script(b"test", b"\x07\x00\x00\x00", n_qm31=1)
    b, _ = orc.channel_script(b"test", b"\x07\x00\x00\x00", n_qm31=1)
    c, _ = orc.channel_script(b"test", b"\x08\x00\x00\x00", n_qm31=1)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
