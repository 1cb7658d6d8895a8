"""Canonical wire encoding (src/core/serialization.zig:58-190, docs/wire.md).

Little-endian integers, ``usize`` as 8 bytes, slices as a u64 length followed by the
elements, optionals as a one-byte presence flag, structs in declaration order, field
elements as their ``SIZE`` little-endian bytes (QM31 = a.c0 | a.c1 | b.c0 | b.c1).
These helpers build the byte buffers the ``zs_m31_*`` C ABI takes and parse the proofs
it returns.
"""
import struct
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

P = 2147483647


def u8(v):
    return struct.pack("<B", v)


def u64(v):
    return struct.pack("<Q", v)


def qm31(v):
    """v: 4 ints (a.c0, a.c1, b.c0, b.c1)."""
    return struct.pack("<4I", *[int(x) for x in v])


def qm31_slice(vals):
    arr = np.ascontiguousarray(np.asarray(vals, dtype=np.uint32).reshape(-1, 4))
    return u64(arr.shape[0]) + arr.tobytes()


def columns(cols):
    """[]const []const QM31: cols is a sequence of (n, 4) uint32 arrays."""
    out = [u64(len(cols))]
    for c in cols:
        out.append(qm31_slice(c))
    return b"".join(out)


def m31_column_as_qm31(col):
    """Embeds an M31 column (n,) into QM31 (n, 4)."""
    col = np.asarray(col, dtype=np.uint32)
    out = np.zeros((col.size, 4), dtype=np.uint32)
    out[:, 0] = col
    return out


@dataclass
class StarkParams:
    """src/m31/stark.zig:75-90."""
    trace_log: int
    log_blowup: int = 3
    num_queries: int = 16
    remainder_log: int = 3

    def encode(self):
        return u8(self.trace_log) + u8(self.log_blowup) + u64(self.num_queries) + u8(self.remainder_log)

    @property
    def n(self):
        return 1 << self.trace_log

    @property
    def N(self):
        return 1 << (self.trace_log + self.log_blowup)


class Reader:
    def __init__(self, data: bytes):
        self.d = data
        self.pos = 0

    def take(self, k):
        if self.pos + k > len(self.d):
            raise ValueError("unexpected end")
        r = self.d[self.pos:self.pos + k]
        self.pos += k
        return r

    def u8(self):
        return self.take(1)[0]

    def u64(self):
        return struct.unpack("<Q", self.take(8))[0]

    def digest(self):
        return self.take(32)

    def qm31(self):
        return struct.unpack("<4I", self.take(16))

    def digests(self):
        return [self.digest() for _ in range(self.u64())]

    def qm31s(self):
        return [self.qm31() for _ in range(self.u64())]

    def end(self):
        if self.pos != len(self.d):
            raise ValueError("trailing bytes")


@dataclass
class FriPair:
    value0: tuple
    value1: tuple
    path0: list
    path1: list


@dataclass
class FriQuery:
    index: int
    pairs: List[FriPair]


@dataclass
class FriProof:
    """src/m31/fri.zig:72-79 (allocator field skipped on the wire)."""
    log_size: int
    log_blowup: int
    num_queries: int
    remainder_log: int
    roots: list
    remainder: list
    queries: List[FriQuery]

    @staticmethod
    def read(r: Reader):
        ls, lb, nq, rl = r.u8(), r.u8(), r.u64(), r.u8()
        roots = r.digests()
        rem = r.qm31s()
        queries = []
        for _ in range(r.u64()):
            idx = r.u64()
            pairs = []
            for _ in range(r.u64()):
                v0, v1 = r.qm31(), r.qm31()
                pairs.append(FriPair(v0, v1, r.digests(), r.digests()))
            queries.append(FriQuery(idx, pairs))
        return FriProof(ls, lb, nq, rl, roots, rem, queries)

    def encode(self):
        out = [u8(self.log_size), u8(self.log_blowup), u64(self.num_queries), u8(self.remainder_log)]
        out.append(u64(len(self.roots)) + b"".join(self.roots))
        out.append(u64(len(self.remainder)) + b"".join(qm31(v) for v in self.remainder))
        out.append(u64(len(self.queries)))
        for q in self.queries:
            out.append(u64(q.index) + u64(len(q.pairs)))
            for p in q.pairs:
                out.append(qm31(p.value0) + qm31(p.value1))
                out.append(u64(len(p.path0)) + b"".join(p.path0))
                out.append(u64(len(p.path1)) + b"".join(p.path1))
        return b"".join(out)


@dataclass
class QueryReveal:
    query_index: int
    values: list
    paths: list


@dataclass
class StarkProof:
    """GenericStark(Air).Proof, src/m31/stark.zig:107-122."""
    params: StarkParams
    trace_roots: list
    preprocessed_roots: Optional[list]
    accumulator_roots: Optional[list]
    quotient_root: bytes
    deep_evals: list
    fri: FriProof
    queries: List[QueryReveal] = field(default_factory=list)

    @staticmethod
    def decode(data: bytes):
        r = Reader(data)
        params = StarkParams(r.u8(), r.u8(), r.u64(), r.u8())
        trace_roots = r.digests()
        pre = r.digests() if r.u8() == 1 else None
        acc = r.digests() if r.u8() == 1 else None
        qroot = r.digest()
        deep = r.qm31s()
        fri = FriProof.read(r)
        queries = []
        for _ in range(r.u64()):
            qi = r.u64()
            vals = r.qm31s()
            paths = [r.digests() for _ in range(r.u64())]
            queries.append(QueryReveal(qi, vals, paths))
        r.end()
        return StarkProof(params, trace_roots, pre, acc, qroot, deep, fri, queries)

    def encode(self):
        out = [self.params.encode()]
        out.append(u64(len(self.trace_roots)) + b"".join(self.trace_roots))
        for opt in (self.preprocessed_roots, self.accumulator_roots):
            out.append(u8(0) if opt is None else u8(1) + u64(len(opt)) + b"".join(opt))
        out.append(self.quotient_root)
        out.append(u64(len(self.deep_evals)) + b"".join(qm31(v) for v in self.deep_evals))
        out.append(self.fri.encode())
        out.append(u64(len(self.queries)))
        for q in self.queries:
            out.append(u64(q.query_index) + u64(len(q.values)) + b"".join(qm31(v) for v in q.values))
            out.append(u64(len(q.paths)))
            for p in q.paths:
                out.append(u64(len(p)) + b"".join(p))
        return b"".join(out)
