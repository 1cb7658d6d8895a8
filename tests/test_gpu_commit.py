"""GPU circle commit workload (circle LDE, row-leaf Merkle tree, gamma combination,
fold chain with per-layer commits) bit-exact against the oracle."""
import numpy as np
import pytest

from zs_b200 import workload as wl

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _inputs(n_cols, log_rows, n_folds, seed):
    rng = np.random.default_rng(seed)
    trace = rng.integers(0, P, (n_cols, 1 << log_rows), dtype=np.uint32)
    gammas = rng.integers(0, P, (n_cols, 4), dtype=np.uint32)
    alphas = rng.integers(0, P, (n_folds, 4), dtype=np.uint32)
    return trace, gammas, alphas


@pytest.mark.parametrize("n_cols,log_rows,log_blowup,n_folds", [
    (1, 1, 1, 1), (1, 2, 1, 2), (3, 3, 2, 4), (8, 6, 2, 6), (16, 10, 2, 8), (64, 12, 2, 10),
    (5, 11, 1, 11), (2, 13, 3, 16), (64, 14, 2, 16), (17, 9, 0, 3), (256, 8, 2, 5)])
def test_commit_matches_oracle(orc, n_cols, log_rows, log_blowup, n_folds):
    from zs_b200 import native
    trace, gammas, alphas = _inputs(n_cols, log_rows, n_folds, 7 * n_cols + log_rows)
    want = orc.circle_commit(trace, log_blowup, gammas, alphas, keep_lde=True)
    plan = native.CommitPlan(n_cols, log_rows, log_blowup, n_folds)
    plan.set_challenges(gammas, alphas)
    plan.upload(trace)
    plan.run()
    got = plan.results()
    assert np.array_equal(plan.lde(), want["lde"])
    assert np.array_equal(plan.layer(0), want["g"])
    assert got["lde_root"] == want["lde_root"]
    assert np.array_equal(got["layer_roots"], want["layer_roots"])
    assert np.array_equal(got["final_layer"], want["final_layer"])
    # a second run on the same plan gives the same bytes
    plan.run()
    again = plan.results()
    assert again["lde_root"] == want["lde_root"]
    plan.close()
    one = native.circle_commit(trace, log_blowup, gammas, alphas)
    assert one["lde_root"] == want["lde_root"]
    assert np.array_equal(one["final_layer"], want["final_layer"])


@pytest.mark.parametrize("log_blowup", [0, 1, 3])
def test_commit_2p20_rows_each_blowup_matches_oracle(orc, log_blowup):
    """2^20 rows run the middle pass's compile-time layout (groups of 2^10 on both
    sides), whose quarter loop runs 2^log_blowup times: the LDE bytes against the oracle
    for one, two and eight quarters (the full-size test covers four)."""
    from zs_b200 import native
    trace, gammas, alphas = _inputs(2, 20, 4, 20 + log_blowup)
    want = orc.circle_commit(trace, log_blowup, gammas, alphas, keep_lde=True)
    plan = native.CommitPlan(2, 20, log_blowup, 4)
    plan.set_challenges(gammas, alphas)
    plan.upload(trace)
    plan.run()
    got = plan.results()
    assert np.array_equal(plan.lde(), want["lde"])
    assert got["lde_root"] == want["lde_root"]
    assert np.array_equal(got["layer_roots"], want["layer_roots"])
    assert np.array_equal(got["final_layer"], want["final_layer"])
    plan.close()


def test_commit_full_size_matches_oracle(orc):
    """The 64 x 2^20 blowup-4 workload with 16 folds (2^22 -> 2^6), seeded inputs."""
    from zs_b200 import native
    trace, gammas, alphas = wl.commit_inputs(64, 20, 16)
    plan = native.CommitPlan(64, 20, 2, 16)
    plan.set_challenges(gammas, alphas)
    plan.upload(trace)
    plan.run()
    got = plan.results()
    want = orc.circle_commit(trace, 2, gammas, alphas)
    assert got["lde_root"] == want["lde_root"]
    assert np.array_equal(got["layer_roots"], want["layer_roots"])
    assert np.array_equal(got["final_layer"], want["final_layer"])
    # size-independent property: the LDE is the extension of a degree < 2^20 circle
    # polynomial, so its inverse transform on the big domain has zero high halves
    lde = plan.lde()
    for c in (0, 63):
        coeffs = native.circle_ifft(lde[c])
        half = 1 << 21
        assert not coeffs[1 << 19:half].any() and not coeffs[half + (1 << 19):].any()
        assert np.array_equal(native.circle_fft(coeffs), lde[c])
    plan.close()


@pytest.mark.parametrize("n_cols,log_rows,log_blowup,n_folds", [(13, 10, 2, 8), (64, 12, 2, 10), (3, 4, 1, 3)])
def test_run_host_matches_oracle(orc, n_cols, log_rows, log_blowup, n_folds):
    """run_host (column groups uploaded from pinned memory while earlier groups' LDE
    runs), twice in a row on the same plan, equals the oracle."""
    import torch
    from zs_b200 import native
    trace, gammas, alphas = _inputs(n_cols, log_rows, n_folds, 11 * n_cols + log_rows)
    want = orc.circle_commit(trace, log_blowup, gammas, alphas)
    pinned = torch.from_numpy(trace.view(np.int32)).pin_memory()
    plan = native.CommitPlan(n_cols, log_rows, log_blowup, n_folds)
    plan.set_challenges(gammas, alphas)
    for _ in range(2):
        plan.run_host(pinned.data_ptr())
        got = plan.results()
        assert got["lde_root"] == want["lde_root"]
        assert np.array_equal(got["layer_roots"], want["layer_roots"])
        assert np.array_equal(got["final_layer"], want["final_layer"])
    plan.close()
