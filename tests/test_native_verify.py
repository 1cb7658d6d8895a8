"""The library's host-side verifier (zs_m31_verify) against oracle proofs: accepts
every valid proof, rejects false statements and tampered proofs, and reports
malformed input with the reference's error codes. Needs no GPU."""
import pytest

from zs_b200 import native, wire
from zs_b200 import workload as wl

P = 2**31 - 1


def _proof(orc, air, params, pi, tr, pre=(), sep=b"v"):
    pre_b = wire.columns(list(pre)) if len(pre) else b""
    return orc.prove(air, params.encode(), pi, pre_b, wire.columns(tr), sep, mode=1)


@pytest.mark.parametrize("trace_log,log_blowup", [(4, 3), (8, 2), (6, 1), (1, 2)])
def test_accepts_fib(orc, trace_log, log_blowup):
    params = wire.StarkParams(trace_log, log_blowup, 16, max(2, min(3, trace_log + log_blowup - 1)))
    tr = wl.fib_trace(1 << trace_log)
    pi = wl.fib_public(tr)
    proof = _proof(orc, wl.AIR_FIB, params, pi, tr)
    assert native.verify(wl.AIR_FIB, params, pi, proof, b"v")
    assert not native.verify(wl.AIR_FIB, params, pi, proof, b"other separator")
    bad_pi = wire.qm31(((int(tr[0][-1][0]) + 1) % P, 0, 0, 0))
    assert not native.verify(wl.AIR_FIB, params, bad_pi, proof, b"v")


@pytest.mark.parametrize("air,gen", [(wl.AIR_RANGE_CHECK, wl.range_check_trace), (wl.AIR_AND_TABLE, wl.and_table_trace),
                                     (wl.AIR_MULTIPLICITY, wl.multiplicity_trace)])
def test_lookup_airs(orc, air, gen):
    params = wire.StarkParams(4, 3, 16, 3)
    tr, table = gen(16)
    proof = _proof(orc, air, params, b"", tr, table)
    assert native.verify(air, params, b"", proof, b"v")
    sp = wire.StarkProof.decode(proof)
    v = sp.queries[0].values[0]
    sp.queries[0].values[0] = ((v[0] + 1) % P,) + tuple(v[1:])
    assert not native.verify(air, params, b"", sp.encode(), b"v")


def test_examples(orc):
    params = wire.StarkParams(3, 3, 16, 3)
    for air, (tr, pi) in ((wl.AIR_RESCUE_EXAMPLE, wl.rescue_example()), (wl.AIR_LINEAR_EXAMPLE, wl.linear_example())):
        proof = _proof(orc, air, params, pi, tr)
        assert native.verify(air, params, pi, proof, b"v")


def test_tampering_each_section(orc):
    params = wire.StarkParams(5, 2, 16, 3)
    tr, pi = wl.seeded_fib(5)
    proof = _proof(orc, wl.AIR_SEEDED_FIB, params, pi, tr)
    assert native.verify(wl.AIR_SEEDED_FIB, params, pi, proof, b"v")
    sp = wire.StarkProof.decode(proof)
    mutations = []
    s = wire.StarkProof.decode(proof); s.trace_roots[0] = bytes(32); mutations.append(s)
    s = wire.StarkProof.decode(proof); s.quotient_root = bytes(32); mutations.append(s)
    s = wire.StarkProof.decode(proof); d = s.deep_evals[0]; s.deep_evals[0] = ((d[0] + 1) % P,) + d[1:]; mutations.append(s)
    s = wire.StarkProof.decode(proof); s.fri.roots[1] = bytes(32); mutations.append(s)
    s = wire.StarkProof.decode(proof); r = s.fri.remainder[0]; s.fri.remainder[0] = ((r[0] + 1) % P,) + r[1:]; mutations.append(s)
    s = wire.StarkProof.decode(proof); s.fri.queries[3].pairs[2].path0[0] = bytes(32); mutations.append(s)
    s = wire.StarkProof.decode(proof); s.queries[5].paths[1][0] = bytes(32); mutations.append(s)
    s = wire.StarkProof.decode(proof); s.queries[2].query_index ^= 1; mutations.append(s)
    for s in mutations:
        assert not native.verify(wl.AIR_SEEDED_FIB, params, pi, s.encode(), b"v")
    assert len(sp.queries) == 16


def test_malformed(orc):
    params = wire.StarkParams(4, 3, 12, 3)
    tr = wl.fib_trace(16)
    pi = wl.fib_public(tr)
    proof = _proof(orc, wl.AIR_FIB, params, pi, tr)
    for bad in (proof[:-1], proof + b"\x00", b""):
        with pytest.raises(native.ZsError) as e:
            native.verify(wl.AIR_FIB, params, pi, bad, b"v")
        assert e.value.code == -2
    with pytest.raises(native.ZsError) as e:
        native.verify(wl.AIR_FIB, params, pi[:-1], proof, b"v")
    assert e.value.code == -2


def test_rescue_stacked(orc):
    tr, pi = wl.rescue_stacked(6)
    params = wire.StarkParams(6, 2, 16, 3)
    proof = _proof(orc, wl.AIR_RESCUE_STACKED, params, pi, tr)
    assert native.verify(wl.AIR_RESCUE_STACKED, params, pi, proof, b"v")
    bad = bytearray(pi)
    bad[70] ^= 1
    assert not native.verify(wl.AIR_RESCUE_STACKED, params, bytes(bad), proof, b"v")


@pytest.mark.parametrize("threads", [1, 3, 0])
def test_verify_batch_matches_single(orc, threads):
    """zs_m31_verify_batch gives each job the single call's answer: valid proofs,
    false statements, tampered and malformed proofs mixed in one batch."""
    jobs = []
    for i, lg in enumerate([3, 4, 5, 6]):
        params = wire.StarkParams(lg, 2, 16, 3)
        tr, pi = wl.seeded_fib(lg, 100 + i)
        proof = _proof(orc, wl.AIR_SEEDED_FIB, params, pi, tr)
        jobs.append((wl.AIR_SEEDED_FIB, params, pi, proof, b"v"))
    tr, pi = wl.rescue_stacked(5)
    params = wire.StarkParams(5, 2, 16, 3)
    jobs.append((wl.AIR_RESCUE_STACKED, params, pi, _proof(orc, wl.AIR_RESCUE_STACKED, params, pi, tr), b"v"))
    a, p, pi0, pr0, s0 = jobs[0]
    bad_pi = bytearray(pi0)
    bad_pi[32] ^= 1
    sp = wire.StarkProof.decode(pr0)
    sp.quotient_root = bytes(32)
    jobs += [(a, p, bytes(bad_pi), pr0, s0), (a, p, pi0, sp.encode(), s0), (a, p, pi0, pr0[:-3], s0),
             (a, p, pi0, pr0, b"other")]
    got = native.verify_batch(jobs, threads=threads)
    want = []
    for j in jobs:
        try:
            want.append(native.verify(*j))
        except native.ZsError as e:
            want.append(e.code)
    assert got == want
    assert got[:5] == [True] * 5 and got[5] is False and got[6] is False and got[7] == -2 and got[8] is False
    assert native.verify_batch([]) == []


def test_rejects_missing_reveals_the_reference_accepts(orc):
    """The reference verifier (stark.zig:713) checks only the reveals a proof carries,
    so a proof with its reveal list cut short, or emptied, passes there on FRI alone.
    The library requires one reveal per FRI query; the oracle (the reference's
    behaviour) still accepts, which pins that this is a deliberate difference."""
    params = wire.StarkParams(5, 2, 16, 3)
    tr, pi = wl.seeded_fib(5)
    proof = _proof(orc, wl.AIR_SEEDED_FIB, params, pi, tr)
    for keep in (0, 7, 15):
        s = wire.StarkProof.decode(proof)
        s.queries = s.queries[:keep]
        cut = s.encode()
        assert not native.verify(wl.AIR_SEEDED_FIB, params, pi, cut, b"v")
        assert orc.verify(wl.AIR_SEEDED_FIB, params.encode(), pi, cut, b"v")


@pytest.mark.parametrize("trace_log", [2, 6])
def test_ml_linear(orc, trace_log):
    """The library verifier's linear-layer composition (ml_composition) accepts the
    oracle's proofs and rejects a changed quotient root or public weight."""
    tr, pre, pi = wl.ml_linear(trace_log)
    params = wire.StarkParams(trace_log, 2, 16, 3)
    proof = _proof(orc, wl.AIR_ML_LINEAR, params, pi, tr, pre)
    assert native.verify(wl.AIR_ML_LINEAR, params, pi, proof, b"v")
    s = wire.StarkProof.decode(proof)
    s.quotient_root = bytes(32)
    assert not native.verify(wl.AIR_ML_LINEAR, params, pi, s.encode(), b"v")
    bad = bytearray(pi)
    bad[8] ^= 1  # W[0][0]
    assert not native.verify(wl.AIR_ML_LINEAR, params, bytes(bad), proof, b"v")
