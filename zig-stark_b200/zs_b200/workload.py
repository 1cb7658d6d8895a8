"""Seeded synthetic inputs and trace generators.

PRNG: SplitMix64. A uniform M31 element takes the top 31 bits of an output and
rejects 2^31 - 1, so values are uniform in [0, p - 1]. A uniform QM31 element is four
uniform M31 words (a.c0, a.c1, b.c0, b.c1). Seeds: 0x5EED0001 (Fibonacci a_1),
0x5EED0002 (commit trace), 0x5EED0003 (column weights gamma), 0x5EED0004 (fold
challenges alpha).

Trace generators follow the reference AIRs' own ``generateTrace`` functions
(src/m31/stark.zig:908-925, 999-1030, 1081-1120, 1173-1205).
"""
from collections import namedtuple

import numpy as np

from . import wire

P = 2147483647
MASK64 = (1 << 64) - 1

AIR_FIB = 0
AIR_SEEDED_FIB = 1
AIR_RANGE_CHECK = 2
AIR_AND_TABLE = 3
AIR_MULTIPLICITY = 4
AIR_RESCUE_EXAMPLE = 5
AIR_LINEAR_EXAMPLE = 6

SEED_FIB = 0x5EED0001
SEED_COMMIT_TRACE = 0x5EED0002
SEED_COMMIT_GAMMA = 0x5EED0003
SEED_COMMIT_ALPHA = 0x5EED0004


def splitmix64(seed: int, count: int) -> np.ndarray:
    """`count` consecutive SplitMix64 outputs from state `seed` (uint64 array)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed & MASK64) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_m31(seed: int, count: int) -> np.ndarray:
    """`count` uniform M31 values in [0, p-1] (top 31 bits, rejecting p)."""
    out = np.empty(0, dtype=np.uint32)
    drawn = 0
    state = seed
    while out.size < count:
        need = count - out.size
        batch = splitmix64(state, need + need // 64 + 16)
        drawn = batch.size
        state = (state + drawn * 0x9E3779B97F4A7C15) & MASK64
        v = (batch >> np.uint64(33)).astype(np.uint32)
        v = v[v != P]
        out = np.concatenate([out, v])
    return out[:count]


def uniform_qm31(seed: int, count: int) -> np.ndarray:
    return uniform_m31(seed, 4 * count).reshape(count, 4)


def qm31_add(a, b):
    return ((np.asarray(a, dtype=np.uint64) + np.asarray(b, dtype=np.uint64)) % P).astype(np.uint32)


# ---------------------------------------------------------------------------
# Trace generators (columns are (n, 4) uint32 QM31 arrays)
# ---------------------------------------------------------------------------

def fib_trace(n, a0=0, a1=1):
    """FibAir.generateTrace (stark.zig:908-925) with configurable a_0, a_1 (M31).

    Vectorised in blocks of B rows: with F the Fibonacci numbers (F(-1) = 1),
    a_(j+t) = F(t-1) a_j + F(t) a_(j+1), so every block follows from its first two
    values, and those follow from the previous block's by the same identity at t = B."""
    x0, y0 = a0 % P, a1 % P
    B = max(1, min(n, 1024))
    F = np.zeros(B + 2, dtype=np.uint64)  # F[k] = F(k - 1), k = 0..B+1
    F[0], F[1] = 1, 0
    for k in range(2, B + 2):
        F[k] = (F[k - 1] + F[k - 2]) % P
    blocks = (n + B - 1) // B
    xs = np.zeros(blocks, dtype=np.uint64)
    ys = np.zeros(blocks, dtype=np.uint64)
    x, y = x0, y0
    fb_1, fb, fb1 = int(F[B]), int(F[B + 1]), int((F[B] + F[B + 1]) % P)  # F(B-1), F(B), F(B+1)
    for k in range(blocks):
        xs[k], ys[k] = x, y
        x, y = (fb_1 * x + fb * y) % P, (fb * x + fb1 * y) % P
    a = ((np.outer(xs, F[:B]) + np.outer(ys, F[1:B + 1])) % P).reshape(-1)[:n]
    b = ((np.outer(xs, F[1:B + 1]) + np.outer(ys, F[2:B + 2])) % P).reshape(-1)[:n]
    return [wire.m31_column_as_qm31(a), wire.m31_column_as_qm31(b)]


def fib_public(trace):
    """FibAir PublicInputs {claimed_fib} = last value of column 0."""
    return wire.qm31(trace[0][-1])


def seeded_fib(trace_log, seed=SEED_FIB):
    """The 2^trace_log Fibonacci workload: a_0 = 1, a_1 uniform M31 from `seed`.

    Returns (trace, public_inputs) for AIR_SEEDED_FIB, PublicInputs {a0, a1, claimed}.
    """
    a1 = int(uniform_m31(seed, 1)[0])
    tr = fib_trace(1 << trace_log, 1, a1)
    pi = wire.qm31((1, 0, 0, 0)) + wire.qm31((a1, 0, 0, 0)) + wire.qm31(tr[0][-1])
    return tr, pi


def range_check_trace(n):
    """RangeCheckAir.generateTrace / generateTable (stark.zig:999-1030)."""
    value = np.zeros(n, dtype=np.uint32)
    mult = np.zeros(n, dtype=np.uint32)
    sel = np.zeros(n, dtype=np.uint32)
    table = np.zeros(n, dtype=np.uint32)
    for i in range(n):
        if i < n // 2:
            value[i], mult[i], sel[i] = i % 4, 1, 1
        else:
            table[i] = i % 4
    cols = [wire.m31_column_as_qm31(c) for c in (value, mult, sel)]
    return cols, [wire.m31_column_as_qm31(table)]


def and_table_trace(n):
    """AndTableAir.generateTrace / generateTable (stark.zig:1081-1120)."""
    x = np.zeros(n, dtype=np.uint32)
    y = np.zeros(n, dtype=np.uint32)
    sel = np.zeros(n, dtype=np.uint32)
    ta = np.zeros(n, dtype=np.uint32)
    tb = np.zeros(n, dtype=np.uint32)
    for i in range(n):
        if i < n // 2:
            x[i], y[i], sel[i] = (i % 4) & 1, (i % 4) >> 1, 1
        else:
            ta[i], tb[i] = (i % 4) & 1, (i % 4) >> 1
    cols = [wire.m31_column_as_qm31(c) for c in (x, y, sel)]
    return cols, [wire.m31_column_as_qm31(ta), wire.m31_column_as_qm31(tb)]


def multiplicity_trace(n):
    """MultiplicityAir.generateTrace / generateTable (stark.zig:1173-1205)."""
    value = np.zeros(n, dtype=np.uint32)
    mult = np.zeros(n, dtype=np.uint32)
    sel = np.zeros(n, dtype=np.uint32)
    table = np.zeros(n, dtype=np.uint32)
    for i in range(n):
        if i < 4:
            value[i], mult[i], sel[i] = i, 3, 1
        else:
            table[i] = i % 4
    cols = [wire.m31_column_as_qm31(c) for c in (value, mult, sel)]
    return cols, [wire.m31_column_as_qm31(table)]


def commit_inputs(n_cols=64, log_rows=20, n_folds=16):
    """The circle commit workload: trace (n_cols, 2^log_rows) uniform M31 (column-major),
    gammas (n_cols, 4), alphas (n_folds, 4) uniform QM31."""
    trace = uniform_m31(SEED_COMMIT_TRACE, n_cols << log_rows).reshape(n_cols, 1 << log_rows)
    gammas = uniform_qm31(SEED_COMMIT_GAMMA, n_cols)
    alphas = uniform_qm31(SEED_COMMIT_ALPHA, n_folds)
    return trace, gammas, alphas


# ---------------------------------------------------------------------------
# Small exact QM31 arithmetic for building example traces (pure Python ints)
# ---------------------------------------------------------------------------

def _cm_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def qm_mul(x, y):
    """QM31 product with j^2 = -i (src/m31/field/qm31.zig:25-33)."""
    a, b = (x[0], x[1]), (x[2], x[3])
    c, d = (y[0], y[1]), (y[2], y[3])
    ab0 = _cm_mul(a, c)
    ab1 = _cm_mul(b, d)
    cross = _cm_mul(((a[0] + b[0]) % P, (a[1] + b[1]) % P), ((c[0] + d[0]) % P, (c[1] + d[1]) % P))
    ra = ((ab0[0] + ab1[1]) % P, (ab0[1] - ab1[0]) % P)  # ab0 - i*ab1
    rb = ((cross[0] - ab0[0] - ab1[0]) % P, (cross[1] - ab0[1] - ab1[1]) % P)
    return (ra[0], ra[1], rb[0], rb[1])


def qm_add(x, y):
    return tuple((u + v) % P for u, v in zip(x, y))


def qm_pow(x, e):
    r = (1, 0, 0, 0)
    while e:
        if e & 1:
            r = qm_mul(r, x)
        x = qm_mul(x, x)
        e >>= 1
    return r


RESCUE_MDS = ((2, 3, 1, 1), (1, 2, 3, 1), (1, 1, 2, 3), (3, 1, 1, 2))


def rescue_round_constants(rounds=7, s=4):
    """examples/rescue/src/main.zig:28-38 (LCG, top bits, embedded M31)."""
    seed = 0x243F6A8885A308D3
    out = []
    for _ in range(rounds):
        row = []
        for _ in range(s):
            seed = (seed * 6364136223846793005 + 1442695040888963407) & MASK64
            v = (seed >> 33) & 0xFFFFFFFF
            row.append((v % P if v >= P else v, 0, 0, 0))
        out.append(row)
    return out


def rescue_apply_round(r, state, rc):
    """examples/rescue/src/main.zig:41-52."""
    boxed = [qm_pow(v, 5) for v in state]
    out = []
    for j in range(4):
        acc = (0, 0, 0, 0)
        for l in range(4):
            acc = qm_add(acc, qm_mul(boxed[l], (RESCUE_MDS[j][l], 0, 0, 0)))
        out.append(qm_add(acc, rc[r][j]))
    return out


def rescue_example(initial=((1, 0, 0, 0), (2, 0, 0, 0), (3, 0, 0, 0), (4, 0, 0, 0))):
    """The rescue example trace (n = 8 states, 7 rounds) and PublicInputs {initial, final}."""
    rc = rescue_round_constants()
    state = [tuple(v) for v in initial]
    rows = []
    for r in range(8):
        rows.append(state)
        if r < 7:
            state = rescue_apply_round(r, state, rc)
    cols = [np.array([rows[r][j] for r in range(8)], dtype=np.uint32) for j in range(4)]
    final = rows[7]
    pi = b"".join(wire.qm31(v) for v in initial) + b"".join(wire.qm31(v) for v in final)
    return cols, pi


def linear_example(x=None):
    """The ml_linear example: y = sum_r (r+1) * x_r over 8 inputs, running-sum trace.

    Returns (trace, public_inputs) with PublicInputs {x: []QM31, claimed_y}.
    """
    if x is None:
        x = [(i + 1, 0, 0, 0) for i in range(8)]
    acc = (0, 0, 0, 0)
    col = []
    for r in range(8):
        acc = qm_add(acc, qm_mul((r + 1, 0, 0, 0), x[r]))
        col.append(acc)
    pi = wire.u64(8) + b"".join(wire.qm31(v) for v in x) + wire.qm31(acc)
    return [np.array(col, dtype=np.uint32)], pi


AIR_RESCUE_STACKED = 7
SEED_RESCUE = 0x5EED0005


def _m31_pow5(v):
    v = v.astype(np.uint64)
    v2 = v * v % P
    return v2 * v2 % P * v % P


def rescue_stacked(trace_log, seed=SEED_RESCUE):
    """Independent Rescue permutations (the example's 7 rounds, 8 rows each) stacked to
    2^trace_log rows; initial states uniform M31 from `seed`. Columns s_0..s_3,
    q_j = s_j^2 and t_j = q_j s_j. Returns (trace, public_inputs) for AIR_RESCUE_STACKED with
    PublicInputs {initial: first permutation's input, final: last permutation's output}."""
    n = 1 << trace_log
    if n < 8:
        raise ValueError("stacked rescue needs at least 8 rows")
    perms = n // 8
    rc = rescue_round_constants()
    state = uniform_m31(seed, 4 * perms).reshape(perms, 4).astype(np.uint64)
    s = np.zeros((perms, 8, 4), dtype=np.uint64)
    for t in range(8):
        s[:, t, :] = state
        if t < 7:
            boxed = _m31_pow5(state)
            new = np.zeros_like(state)
            for j in range(4):
                acc = np.zeros(perms, dtype=np.uint64)
                for l in range(4):
                    acc = (acc + boxed[:, l] * RESCUE_MDS[j][l]) % P
                new[:, j] = (acc + rc[t][j][0]) % P
            state = new
    flat = s.reshape(n, 4)
    cols = [wire.m31_column_as_qm31(flat[:, j]) for j in range(4)]
    sq = flat * flat % P
    cols += [wire.m31_column_as_qm31(sq[:, j]) for j in range(4)]
    cols += [wire.m31_column_as_qm31(sq[:, j] * flat[:, j] % P) for j in range(4)]
    initial = [(int(flat[0, j]), 0, 0, 0) for j in range(4)]
    final = [(int(flat[n - 1, j]), 0, 0, 0) for j in range(4)]
    pi = b"".join(wire.qm31(v) for v in initial) + b"".join(wire.qm31(v) for v in final)
    return cols, pi


# ---------------------------------------------------------------------------
# One linear layer y = W x over a batch of input vectors (AIR_ML_LINEAR)
# ---------------------------------------------------------------------------

AIR_ML_LINEAR = 8
SEED_ML_LINEAR = 0x5EED0006
ML_DIM = 128


def uniform_below(seed, count, bound):
    """`count` values uniform in [0, bound) for a power-of-two bound (top bits of
    SplitMix64 outputs)."""
    shift = 64 - (int(bound).bit_length() - 1)
    return (splitmix64(seed, count) >> np.uint64(shift)).astype(np.uint32)


def ml_linear(trace_log, seed=SEED_ML_LINEAR, vectors=None):
    """The linear-layer workload: W (128 x 128) and 2^(trace_log - 1) input vectors,
    entries uniform in [0, 2^16) (W from `seed`, the inputs from seed + 1).

    Rows [0, V) hold the input vectors (sel = 1, mult = 1) with y = W x mod p; rows
    [V, n) are the input table's rows (sel = 0, x = y = 0), where the preprocessed
    columns P_0..P_127 hold the same vectors. The LogUp relation then matches every
    input vector with its table row. Returns (trace, preprocessed, public_inputs) with
    PublicInputs {w: []QM31}."""
    n = 1 << trace_log
    V = vectors if vectors is not None else n // 2
    if not 0 < V <= n // 2:
        raise ValueError("at most half the rows hold input vectors")
    D = ML_DIM
    W = uniform_below(seed, D * D, 1 << 16).reshape(D, D)
    X = uniform_below(seed + 1, V * D, 1 << 16).reshape(V, D)
    Y = (X.astype(np.uint64) @ W.T.astype(np.uint64)) % P  # < 128 * 2^32: exact in u64
    x_cols = np.zeros((D, n), dtype=np.uint32)
    y_cols = np.zeros((D, n), dtype=np.uint32)
    p_cols = np.zeros((D, n), dtype=np.uint32)
    x_cols[:, :V] = X.T
    y_cols[:, :V] = Y.T.astype(np.uint32)
    p_cols[:, n - V:] = X.T
    sel = np.zeros(n, dtype=np.uint32)
    sel[:V] = 1
    trace = [wire.m31_column_as_qm31(c) for c in x_cols] + [wire.m31_column_as_qm31(c) for c in y_cols]
    trace += [wire.m31_column_as_qm31(sel), wire.m31_column_as_qm31(sel.copy())]
    pre = [wire.m31_column_as_qm31(c) for c in p_cols]
    pi = wire.qm31_slice(wire.m31_column_as_qm31(W.reshape(-1)))
    return trace, pre, pi


# ---------------------------------------------------------------------------
# Mixed-size proof streams (batched and served proving)
# ---------------------------------------------------------------------------

SEED_BATCH = 0x5EED0007
SEED_SERVE = 0x5EED0008


def _mix(seed, index):
    return int(splitmix64((seed ^ (index * 0xD1B54A32D192ED03)) & MASK64, 1)[0])


class ProofJob(namedtuple("ProofJob", "air params pi trace sep pre")):
    """One proof request in wire form: AIR id, StarkParams, public inputs, trace columns,
    channel separator and preprocessed columns (b"" when the AIR has none)."""


def proof_job(air, trace_log, seed, sep, num_queries=16, remainder_log=3):
    """One proof request at blowup 4 (a ProofJob)."""
    pre = b""
    if air == AIR_SEEDED_FIB:
        tr, pi = seeded_fib(trace_log, seed)
    elif air == AIR_RESCUE_STACKED:
        tr, pi = rescue_stacked(trace_log, seed)
    elif air == AIR_ML_LINEAR:
        tr, pre_cols, pi = ml_linear(trace_log, seed)
        pre = wire.columns(pre_cols)
    else:
        raise ValueError(f"no stream generator for AIR {air}")
    params = wire.StarkParams(trace_log, 2, num_queries, remainder_log).encode()
    return ProofJob(air, params, pi, wire.columns(tr), sep, pre)


def batch_shapes(count, seed=SEED_BATCH, log_min=10, log_max=20):
    """(air, trace_log, trace seed, channel separator) of `count` independent traces:
    Fibonacci or stacked Rescue 50/50, log2 rows uniform in [log_min, log_max], a
    distinct channel separator per trace."""
    out = []
    for i in range(count):
        r = _mix(seed, i)
        air = AIR_SEEDED_FIB if r & 1 else AIR_RESCUE_STACKED
        lg = log_min + ((r >> 8) % (log_max - log_min + 1))
        out.append((air, lg, (r >> 20) & MASK64, b"zs-batch:%d" % i))
    return out


ML_LINEAR_MAX_LOG = 15  # 2^14 input vectors: the linear layer's full size


def serve_shapes(count, seed=SEED_SERVE, log_min=12, log_max=22, p_geo=0.5, mix=(0.5, 0.3, 0.2)):
    """Served-stream requests: AIR by `mix` (Fibonacci, stacked Rescue, linear layer),
    log2 rows from a geometric distribution (success probability p_geo) truncated to
    [log_min, log_max]. A linear-layer request holds 2^(rows - 1) input vectors of 387
    committed columns, so its rows are capped at 2^15 (2^14 vectors, the layer's full
    size)."""
    out = []
    span = log_max - log_min + 1
    w = np.array([(1 - p_geo) ** k * p_geo for k in range(span)])
    cdf = np.cumsum(w / w.sum())
    edges = np.cumsum(np.asarray(mix, dtype=np.float64) / sum(mix))
    airs = (AIR_SEEDED_FIB, AIR_RESCUE_STACKED, AIR_ML_LINEAR)
    for i in range(count):
        r = _mix(seed, i)
        u = ((r >> 11) & ((1 << 53) - 1)) / float(1 << 53)
        lg = log_min + int(np.searchsorted(cdf, u, side="right"))
        lg = min(lg, log_max)
        v = (r & 0x3FF) / 1024.0
        air = airs[min(int(np.searchsorted(edges, v, side="right")), len(mix) - 1)]
        if air == AIR_ML_LINEAR:
            lg = min(lg, ML_LINEAR_MAX_LOG)
        out.append((air, lg, _mix(seed ^ 0xABCDEF, i), b"zs-serve:%d" % i))
    return out
