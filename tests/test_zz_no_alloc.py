"""The allocation-free circle LDE entry point (zs_m31_circle_lde_noalloc).

It serves callers that cannot call cudaMalloc (a plugin whose host process reserves
all device memory up front in its own arena, or a latency-bound loop where an
allocation may synchronize the device). The test calls it twice in a row through the
C ABI on caller-owned device buffers and checks each output bit for bit against the
low-degree extension of the existing entry point (zs_m31_commit_plan) and against the
oracle's LDE, checks that the second call leaves the device's free memory unchanged,
and checks that a request above its fixed scratch size is rejected. This file is
collected last so that a run stopping at the first failure has already run every
other test.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _plan_lde(trace, log_blowup):
    from zs_b200 import native
    n_cols, n = trace.shape
    plan = native.CommitPlan(n_cols, n.bit_length() - 1, log_blowup, 0)
    plan.set_challenges(np.zeros((n_cols, 4), dtype=np.uint32), None)
    plan.upload(trace)
    plan.run()
    out = plan.lde()
    plan.close()
    return out


def _oracle_lde(trace, log_blowup):
    n_cols = trace.shape[0]
    res = oracle.circle_commit(trace, log_blowup, np.zeros((n_cols, 4), dtype=np.uint32),
                               np.zeros((0, 4), dtype=np.uint32), keep_lde=True)
    return res["lde"]


def test_noalloc_lde_matches_plan_and_oracle_on_two_calls():
    import torch
    from zs_b200 import native
    cases = [(4, 12, 2), (3, 9, 3)]
    rng = np.random.default_rng(77)
    traces = [rng.integers(0, P, (c, 1 << l), dtype=np.uint32) for c, l, _ in cases]
    bufs = []
    for (c, l, b), tr in zip(cases, traces):
        d_in = torch.from_numpy(tr.view(np.int32)).cuda()
        d_out = torch.empty((c, 1 << (l + b)), dtype=torch.int32, device="cuda")
        bufs.append((d_in, d_out))
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free_before = None
    for k, ((c, l, b), (d_in, d_out)) in enumerate(zip(cases, bufs)):
        rc = native.circle_lde_noalloc(d_in.data_ptr(), d_out.data_ptr(), c, l, b, stream)
        assert rc == 0
        torch.cuda.synchronize()
        if k == 0:
            # the first call on the device backs the scratch array; later calls allocate nothing
            free_before = torch.cuda.mem_get_info()[0]
    assert torch.cuda.mem_get_info()[0] == free_before
    for (c, l, b), tr, (_, d_out) in zip(cases, traces, bufs):
        got = d_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, _oracle_lde(tr, b))
        assert np.array_equal(got, _plan_lde(tr, b))


def test_noalloc_rejects_sizes_above_its_scratch():
    import torch
    from zs_b200 import native
    d = torch.empty(4, dtype=torch.int32, device="cuda")
    # 1 column of 2^20 rows at blowup 4 needs 2^21 + 2^23 + 2^20 + 2^22 words > 2^22
    assert native.circle_lde_noalloc(d.data_ptr(), d.data_ptr(), 1, 20, 2) == -2
