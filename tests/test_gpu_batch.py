"""Batched and served proving (zs_m31_prove_batch, zs_m31_server_*): every proof in a
mixed batch or a served stream is byte-identical to the same job proven alone, and
the oracle's proof of that job."""
import numpy as np
import pytest

from zs_b200 import wire
from zs_b200 import workload as wl

pytestmark = pytest.mark.gpu


def _mixed_jobs():
    jobs = []
    for i, (air, lg) in enumerate([(wl.AIR_SEEDED_FIB, 10), (wl.AIR_RESCUE_STACKED, 6), (wl.AIR_SEEDED_FIB, 4),
                                   (wl.AIR_RESCUE_STACKED, 11), (wl.AIR_SEEDED_FIB, 13), (wl.AIR_RESCUE_STACKED, 3),
                                   (wl.AIR_SEEDED_FIB, 7), (wl.AIR_RESCUE_STACKED, 9), (wl.AIR_ML_LINEAR, 5),
                                   (wl.AIR_ML_LINEAR, 8)]):
        jobs.append(wl.proof_job(air, lg, 1000 + i, b"zig-stark:test:" + bytes([i])))
    tr, table = wl.range_check_trace(64)
    jobs.append((wl.AIR_RANGE_CHECK, wire.StarkParams(6, 2, 16, 3).encode(), b"", wire.columns(tr),
                 b"zig-stark:stark:lookup", wire.columns(table)))
    return jobs


def _alone(job):
    from zs_b200 import native
    air, params, pi, trace, sep = job[:5]
    pre = job[5] if len(job) > 5 else b""
    return native.prove(air, params, pi, trace, pre, sep)


def _as_kwargs(job):
    air, params, pi, trace, sep = job[:5]
    return dict(air_id=air, params=params, public_inputs=pi, trace=trace,
                preprocessed=job[5] if len(job) > 5 else b"", channel_sep=sep)


@pytest.mark.parametrize("concurrency", [1, 4, 16])
def test_batch_matches_alone(orc, concurrency):
    from zs_b200 import native
    jobs = _mixed_jobs()
    got = native.prove_batch([_as_kwargs(j) for j in jobs], concurrency=concurrency)
    for j, g in zip(jobs, got):
        assert isinstance(g, bytes)
        assert g == _alone(j)
    # two of them against the oracle as well
    for j, g in [(jobs[0], got[0]), (jobs[1], got[1]), (jobs[8], got[8])]:
        air, params, pi, trace, sep, pre = j
        assert g == orc.prove(air, params, pi, pre, trace, sep, mode=1)
        assert orc.verify(air, params, pi, g, sep)


def test_batch_tight_budget_runs_one_at_a_time():
    from zs_b200 import native
    jobs = _mixed_jobs()[:4]
    got = native.prove_batch([_as_kwargs(j) for j in jobs], concurrency=4, hbm_budget=1)
    assert got == [_alone(j) for j in jobs]


def test_batch_isolates_failing_job():
    from zs_b200 import native
    jobs = [_as_kwargs(j) for j in _mixed_jobs()[:3]]
    bad = dict(jobs[1])
    bad["public_inputs"] = b"\x00" * 5  # malformed PublicInputs
    short = dict(jobs[2])
    short["params"] = b"\x04"  # truncated StarkParams
    got = native.prove_batch([jobs[0], bad, short, jobs[0]], concurrency=3)
    assert got[1] == -2 and got[2] == -2
    assert isinstance(got[0], bytes) and got[0] == got[3]


def test_batch_empty():
    from zs_b200 import native
    assert native.prove_batch([]) == []


def test_server_stream_matches_alone():
    """Requests submitted while others are on the device (continuous batching): each
    result equals the proof of the same job alone."""
    from zs_b200 import native
    jobs = _mixed_jobs()
    want = [_alone(j) for j in jobs]
    with native.Server(workers=4) as srv:
        first = [srv.submit(**_as_kwargs(j)) for j in jobs[:4]]
        # the rest arrive after the first requests are in flight
        got = {}
        t0 = first[0]
        got[0] = srv.poll(t0, wait=True)
        rest = [srv.submit(**_as_kwargs(j)) for j in jobs[4:]]
        tickets = first + rest
        for k, t in enumerate(tickets):
            if k == 0:
                continue
            got[k] = srv.poll(t, wait=True)
        for k in range(len(jobs)):
            proof, latency = got[k]
            assert proof == want[k]
            assert latency > 0
        with pytest.raises(native.ZsError) as e:
            srv.poll(tickets[0])  # released by the poll that returned it
        assert e.value.code == -2


def test_server_poll_without_wait():
    from zs_b200 import native
    job = wl.proof_job(wl.AIR_SEEDED_FIB, 12, 7, b"zig-stark:test:nowait")
    with native.Server(workers=1) as srv:
        t = srv.submit(**_as_kwargs(job))
        r = srv.poll(t, wait=False)
        while r is None:
            r = srv.poll(t, wait=False)
        assert r[0] == _alone(job)


def test_server_failing_request():
    from zs_b200 import native
    job = _as_kwargs(_mixed_jobs()[0])
    job["public_inputs"] = b"\x01"
    with native.Server(workers=2) as srv:
        t = srv.submit(**job)
        proof, _ = srv.poll(t)
        assert proof == -2
