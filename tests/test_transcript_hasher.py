"""The library's incremental Blake3 (the Fiat-Shamir transcript's hash, csrc/blake3.cuh)
against the `blake3` module: random absorb sequences of bytes and words at every
alignment, across block and chunk boundaries (multi-chunk states with a deep subtree
stack), with the digest of the state and of the state extended by a suffix (how a
sample is drawn: from a snapshot on the host, with finalize_suffix on the device)
checked at random points. Host build of the same header that the
device transcript steps compile."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
blake3 = pytest.importorskip("blake3")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("hasher") / "transcript_hasher")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "zig-stark_b200", "csrc"),
                    os.path.join(ROOT, "tests", "transcript_hasher.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("seed", range(6))
def test_incremental_hasher_matches_blake3(driver, seed):
    rng = np.random.default_rng(seed)
    msg = bytearray()
    ops, want = [], []
    target = int(rng.choice([300, 1100, 5000, 20000]))
    while len(msg) < target:
        kind = rng.integers(0, 4)
        if kind == 0:  # bytes, any length
            n = int(rng.integers(0, 70))
            b = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
            ops.append(f"B {n} {b.hex()}")
            msg += b
        elif kind == 1:  # words
            n = int(rng.integers(1, 12))
            w = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
            ops.append(f"W {n} " + " ".join(f"{int(x):x}" for x in w))
            msg += w.astype("<u4").tobytes()
        elif kind == 2:  # a sample: 6 suffix words
            w = rng.integers(0, 2**32, 6, dtype=np.uint64).astype(np.uint32)
            ops.append("S 6 " + " ".join(f"{int(x):x}" for x in w))
            want += [blake3.blake3(bytes(msg) + w.astype("<u4").tobytes()).hexdigest()] * 2
        else:
            ops.append("F")
            want.append(blake3.blake3(bytes(msg)).hexdigest())
    # land exactly on chunk boundaries and just short of them, then sample
    for pad in (1024 - len(msg) % 1024, 1021, 3, 1024):
        b = bytes(rng.integers(0, 256, pad, dtype=np.uint8))
        ops.append(f"B {pad} {b.hex()}")
        msg += b
        w = [0x2D67697A, 0x72617473, 0x61733A6B, 0x656C706D, 7, 0]
        ops.append("S 6 " + " ".join(f"{x:x}" for x in w))
        want += [blake3.blake3(bytes(msg) + struct.pack("<6I", *w)).hexdigest()] * 2
        ops.append("F")
        want.append(blake3.blake3(bytes(msg)).hexdigest())
    out = subprocess.run([driver], input="\n".join(ops) + "\n", capture_output=True, text=True, check=True)
    assert out.stdout.split() == want
