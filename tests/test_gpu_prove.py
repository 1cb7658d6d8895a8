"""GPU prover (zs_m31_prove) byte-identical to the oracle's GenericStark proofs, and
accepted by the oracle verifier, for every compiled-in AIR."""
import numpy as np
import pytest

from zs_b200 import wire
from zs_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _check(orc, air, params, pi, trace, pre=(), sep=b"s", valid=True):
    from zs_b200 import native
    pre_b = wire.columns(list(pre)) if len(pre) else b""
    got = native.prove(air, params, pi, trace, pre_b, sep)
    want = orc.prove(air, params.encode(), pi, pre_b, wire.columns(trace), sep, mode=1)
    assert got == want
    assert orc.verify(air, params.encode(), pi, got, sep) == valid
    return got


@pytest.mark.parametrize("trace_log,log_blowup,nq,rem", [(4, 3, 12, 3), (8, 3, 16, 3), (1, 2, 4, 2), (2, 1, 8, 2),
                                                         (6, 2, 16, 3), (10, 1, 20, 4), (12, 2, 16, 3)])
def test_fib(orc, trace_log, log_blowup, nq, rem):
    tr = wl.fib_trace(1 << trace_log)
    _check(orc, wl.AIR_FIB, wire.StarkParams(trace_log, log_blowup, nq, rem), wl.fib_public(tr), tr,
           sep=b"zig-stark:stark:fib")


def test_fib_wrong_claim_still_proves(orc):
    # the prover does not check the statement; the verifier rejects (stark.zig:1282-1299)
    tr = wl.fib_trace(16)
    bad = wire.qm31(((int(tr[0][-1][0]) + 1) % wl.P, 0, 0, 0))
    _check(orc, wl.AIR_FIB, wire.StarkParams(4, 3, 12, 3), bad, tr, sep=b"zig-stark:stark:fib", valid=False)


def test_seeded_fib_config(orc):
    """The 2^12-row Fibonacci workload: a_0 = 1, seeded a_1, blowup 4, 16 queries."""
    tr, pi = wl.seeded_fib(12)
    _check(orc, wl.AIR_SEEDED_FIB, wire.StarkParams(12, 2, 16, 3), pi, tr, sep=b"zig-stark:fibonacci:example")


@pytest.mark.parametrize("air,gen", [(wl.AIR_RANGE_CHECK, wl.range_check_trace), (wl.AIR_AND_TABLE, wl.and_table_trace),
                                     (wl.AIR_MULTIPLICITY, wl.multiplicity_trace)])
@pytest.mark.parametrize("trace_log,log_blowup", [(4, 3), (6, 2), (11, 2)])
def test_lookup_airs(orc, air, gen, trace_log, log_blowup):
    tr, table = gen(1 << trace_log)
    valid = air != wl.AIR_MULTIPLICITY or trace_log == 4
    _check(orc, air, wire.StarkParams(trace_log, log_blowup, 16, 3), b"", tr, table, sep=b"zig-stark:stark:lookup",
           valid=valid)


def test_rescue_example(orc):
    tr, pi = wl.rescue_example()
    _check(orc, wl.AIR_RESCUE_EXAMPLE, wire.StarkParams(3, 3, 16, 3), pi, tr, sep=b"zig-stark:rescue:example")


def test_linear_example(orc):
    tr, pi = wl.linear_example()
    _check(orc, wl.AIR_LINEAR_EXAMPLE, wire.StarkParams(3, 3, 16, 3), pi, tr, sep=b"zig-stark:ml_linear:example")


def test_random_qm31_trace(orc):
    # non-embedded QM31 trace values (the prover does not assume M31 inputs)
    rng = np.random.default_rng(9)
    tr = [rng.integers(0, wl.P, (64, 4), dtype=np.uint32) for _ in range(2)]
    _check(orc, wl.AIR_FIB, wire.StarkParams(6, 2, 16, 3), wire.qm31((5, 6, 7, 8)), tr, valid=False)


def test_malformed_inputs(orc):
    from zs_b200 import native
    tr = wl.fib_trace(16)
    params = wire.StarkParams(4, 3, 12, 3)
    with pytest.raises(native.ZsError) as e:
        native.prove(wl.AIR_FIB, params, b"\x00" * 15, tr)
    assert e.value.code == -2
    with pytest.raises(native.ZsError) as e:
        native.prove(wl.AIR_FIB, params, wl.fib_public(tr), tr[:1])
    assert e.value.code == -2
    with pytest.raises(native.ZsError) as e:
        native.prove(wl.AIR_FIB, wire.StarkParams(4, 3, 12, 7), wl.fib_public(tr), tr)
    assert e.value.code == -4
    with pytest.raises(native.ZsError) as e:
        native.prove(99, params, b"", tr)
    assert e.value.code == -1


@pytest.mark.parametrize("trace_log,log_blowup,n_cols", [(0, 1, 1), (3, 2, 2), (10, 2, 5), (14, 1, 3), (16, 2, 2)])
def test_commit_columns(orc, trace_log, log_blowup, n_cols):
    """zs_m31_commit_columns = the per-column trees of stark.zig:397-414."""
    from zs_b200 import native
    rng = np.random.default_rng(trace_log * 7 + n_cols)
    cols = [rng.integers(0, wl.P, (1 << trace_log, 4), dtype=np.uint32) for _ in range(n_cols)]
    b = wire.columns(cols)
    assert native.commit_columns(b, trace_log, log_blowup) == orc.commit_columns(b, n_cols, trace_log, log_blowup)


def test_gpu_proofs_verify_with_library_verifier(orc):
    from zs_b200 import native
    tr, pi = wl.seeded_fib(10)
    params = wire.StarkParams(10, 2, 16, 3)
    proof = native.prove(wl.AIR_SEEDED_FIB, params, pi, tr, b"", b"lib")
    assert native.verify(wl.AIR_SEEDED_FIB, params, pi, proof, b"lib")


@pytest.mark.parametrize("trace_log", [3, 6, 10, 14])
def test_rescue_stacked(orc, trace_log):
    tr, pi = wl.rescue_stacked(trace_log)
    _check(orc, wl.AIR_RESCUE_STACKED, wire.StarkParams(trace_log, 2, 16, 3), pi, tr, sep=b"zig-stark:rescue:example")


def test_rescue_stacked_full_size(orc):
    """2^18 rows of stacked Rescue permutations (2^15 of them) at blowup 4."""
    tr, pi = wl.rescue_stacked(18)
    _check(orc, wl.AIR_RESCUE_STACKED, wire.StarkParams(18, 2, 16, 3), pi, tr, sep=b"zig-stark:rescue:example")


def test_packed_upload_paths(orc):
    """Traces of 4 MiB or more cross PCIe packed (the low word of each element): an M31
    column with raw words at and above p (reduced like M31.fromBytes) next to a column of
    general QM31 values (uploaded whole again), against the oracle."""
    rng = np.random.default_rng(17)
    n = 1 << 17
    m31_col = np.zeros((n, 4), dtype=np.uint32)
    m31_col[:, 0] = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)  # some >= p
    m31_col[:4, 0] = [wl.P, wl.P + 1, 2**32 - 1, 0]
    qm_col = rng.integers(0, wl.P, (n, 4), dtype=np.uint32)
    _check(orc, wl.AIR_FIB, wire.StarkParams(17, 1, 8, 3), wire.qm31((1, 2, 3, 4)), [m31_col, qm_col], valid=False)


def test_grouped_upload_with_preprocessed_columns(orc):
    """2^18 rows of the AND-table lookup AIR: 2 preprocessed + 3 main columns of 4 MiB
    each go up in column groups on a copy stream, the first group holding both
    preprocessed columns and two main ones; against the oracle."""
    tr, table = wl.and_table_trace(1 << 18)
    _check(orc, wl.AIR_AND_TABLE, wire.StarkParams(18, 1, 8, 3), b"", tr, table, sep=b"zig-stark:stark:lookup")


def test_context_prove_matches_prove():
    """zs_m31_prove_ctx on two contexts of device 0, driven from two threads at once,
    gives the bytes of zs_m31_prove for every job."""
    import threading
    from zs_b200 import native
    jobs = [wl.proof_job(air, lg, 5, b"ctx") for air, lg in
            [(wl.AIR_SEEDED_FIB, 10), (wl.AIR_RESCUE_STACKED, 12), (wl.AIR_SEEDED_FIB, 14), (wl.AIR_RESCUE_STACKED, 16)]]
    want = [native.prove(j[0], j[1], j[2], j[3], b"", j[4]) for j in jobs]
    got = [None] * len(jobs)
    with native.Context(0) as c0, native.Context(0) as c1:
        assert c0.device == 0 and c1.device == 0

        def run(ctx, idx):
            for i in idx:
                j = jobs[i]
                got[i] = ctx.prove(j[0], j[1], j[2], j[3], b"", j[4])

        ts = [threading.Thread(target=run, args=(c0, [0, 2])), threading.Thread(target=run, args=(c1, [1, 3]))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    assert got == want


def test_context_rejects_bad_device():
    from zs_b200 import native
    with pytest.raises(native.ZsError) as e:
        native.Context(1 << 20)
    assert e.value.code == -5


def test_maximum_size_proof_verifies():
    """The largest domain the prover takes: 2^24 rows at blowup 4 (2^26 points). Too
    large for the oracle prover in test time, so the proof is checked by the library's
    verifier, a flipped byte must make it fail, and one size more is refused up front."""
    from zs_b200 import native
    tr, pi = wl.seeded_fib(24)
    params = wire.StarkParams(24, 2, 16, 3)
    proof = native.prove(wl.AIR_SEEDED_FIB, params, pi, tr, b"", b"max")
    assert native.verify(wl.AIR_SEEDED_FIB, params, pi, proof, b"max")
    bad = bytearray(proof)
    bad[len(bad) // 2] ^= 1
    try:
        ok = native.verify(wl.AIR_SEEDED_FIB, params, pi, bytes(bad), b"max")
    except native.ZsError:
        ok = False
    assert not ok
    with pytest.raises(native.ZsError) as e:
        native.prove(wl.AIR_SEEDED_FIB, wire.StarkParams(25, 2, 16, 3), pi, tr, b"", b"max")
    assert e.value.code == -2


@pytest.mark.parametrize("air,trace_log", [(wl.AIR_RESCUE_STACKED, 16), (wl.AIR_RESCUE_STACKED, 18),
                                           (wl.AIR_AND_TABLE, 16), (wl.AIR_SEEDED_FIB, 18)])
def test_prover_is_deterministic(orc, air, trace_log):
    """The same job proven three times, on fresh buffers each time and with other
    proofs in between, gives the same bytes (the quotient kernel reads per-thread
    column arrays at indices taken from device memory; the host checks every such
    index before the launch). The first proof is also checked against the oracle."""
    from zs_b200 import native
    if air == wl.AIR_AND_TABLE:
        tr, pre = wl.and_table_trace(1 << trace_log)
        pi = b""
        pre_b = wire.columns(list(pre))
    else:
        tr, pi = wl.rescue_stacked(trace_log) if air == wl.AIR_RESCUE_STACKED else wl.seeded_fib(trace_log)
        pre_b = b""
    params = wire.StarkParams(trace_log, 2 if air != wl.AIR_AND_TABLE else 1, 16, 3)
    first = native.prove(air, params, pi, tr, pre_b, b"det")
    other_tr, other_pi = wl.seeded_fib(12)
    for _ in range(2):
        native.prove(wl.AIR_SEEDED_FIB, wire.StarkParams(12, 2, 16, 3), other_pi, other_tr, b"", b"other")
        assert native.prove(air, params, pi, tr, pre_b, b"det") == first
    if trace_log <= 16:
        assert first == orc.prove(air, params.encode(), pi, pre_b, wire.columns(tr), b"det", mode=1)


@pytest.mark.parametrize("air,trace_log,log_blowup,rem", [(wl.AIR_FIB, 8, 4, 4), (wl.AIR_FIB, 6, 5, 5),
                                                          (wl.AIR_SEEDED_FIB, 12, 4, 5), (wl.AIR_RESCUE_STACKED, 10, 4, 5),
                                                          (wl.AIR_RESCUE_STACKED, 8, 6, 7), (wl.AIR_RANGE_CHECK, 8, 5, 6),
                                                          (wl.AIR_FIB, 2, 12, 12)])
def test_blowups_above_8(orc, air, trace_log, log_blowup, rem):
    """StarkParams.log_blowup is any u8 in the reference (stark.zig:75-90): blowups of
    16 to 4096 prove byte-equal to the oracle and verify."""
    from zs_b200 import native
    pre = ()
    if air == wl.AIR_FIB:
        tr = wl.fib_trace(1 << trace_log)
        pi = wl.fib_public(tr)
    elif air == wl.AIR_SEEDED_FIB:
        tr, pi = wl.seeded_fib(trace_log)
    elif air == wl.AIR_RESCUE_STACKED:
        tr, pi = wl.rescue_stacked(trace_log)
    else:
        tr, pre = wl.range_check_trace(1 << trace_log)
        pi = b""
    params = wire.StarkParams(trace_log, log_blowup, 16, rem)
    proof = _check(orc, air, params, pi, tr, pre, sep=b"blowup")
    assert native.verify(air, params, pi, proof, b"blowup")


@pytest.mark.parametrize("trace_log", [2, 5, 8, 12])
def test_ml_linear(orc, trace_log):
    """The linear layer y = W x (W 128 x 128, inputs bound to the preprocessed input
    table by LogUp) at growing batch sizes, against the oracle."""
    from zs_b200 import native
    tr, pre, pi = wl.ml_linear(trace_log)
    params = wire.StarkParams(trace_log, 2, 16, 3)
    proof = _check(orc, wl.AIR_ML_LINEAR, params, pi, tr, pre, sep=b"zig-stark:ml_linear:layer")
    assert native.verify(wl.AIR_ML_LINEAR, params, pi, proof, b"zig-stark:ml_linear:layer")


def test_ml_linear_full_size(orc):
    """The full layer: W 128 x 128 with entries in [0, 2^16), 2^14 input vectors with
    entries in [0, 2^16) (2^15 rows: the vectors and the input table), blowup 4;
    byte-equal to the oracle, accepted by the oracle and the library verifiers."""
    from zs_b200 import native
    tr, pre, pi = wl.ml_linear(15)
    params = wire.StarkParams(15, 2, 16, 3)
    proof = _check(orc, wl.AIR_ML_LINEAR, params, pi, tr, pre, sep=b"zig-stark:ml_linear:layer")
    assert native.verify(wl.AIR_ML_LINEAR, params, pi, proof, b"zig-stark:ml_linear:layer")


def test_ml_linear_false_statements_fail(orc):
    """A wrong output, or an input vector missing from the input table, still proves
    (the prover does not check the statement) but the proof is rejected, with the same
    bytes as the oracle's."""
    from zs_b200 import native
    tr, pre, pi = wl.ml_linear(6)
    params = wire.StarkParams(6, 2, 16, 3)
    bad_y = [c.copy() for c in tr]
    bad_y[wl.ML_DIM + 3][2, 0] = (int(bad_y[wl.ML_DIM + 3][2, 0]) + 1) % wl.P
    bad_x = [c.copy() for c in pre]
    bad_x[7][-1, 0] = (int(bad_x[7][-1, 0]) + 1) % wl.P  # the table no longer holds the last input vector
    for t, p_ in ((bad_y, pre), (tr, bad_x)):
        proof = _check(orc, wl.AIR_ML_LINEAR, params, pi, t, p_, sep=b"ml", valid=False)
        assert not native.verify(wl.AIR_ML_LINEAR, params, pi, proof, b"ml")
