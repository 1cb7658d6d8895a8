"""Command line: prove synthetic traces on the GPU (for timing and profiling runs).

    PYTHONPATH=zig-stark_b200 python -m zs_b200.cli --air rescue_stacked --log-rows 18 --repeat 2

proves the same job `repeat` times through zs_m31_prove and prints the proof size and
the wall time of each call. The job is `workload.proof_job(air, log_rows, seed, sep)`:
blowup 4, 16 queries, remainder_log 3.

    PYTHONPATH=zig-stark_b200 python -m zs_b200.cli --sumcheck gf8 --log-rows 22 --repeat 1

runs one Binius sum-check round (the values hook, zs_binius_sumcheck_values_gf256 or
_gf128) over three seeded tables of 2^log_rows elements with the terms t0 t1 t2 + 2 t0,
`repeat` times, and prints the values and the wall time of each call.

    PYTHONPATH=zig-stark_b200 python -m zs_b200.cli --commit-cols 16 --log-rows 20 --repeat 2

commits `workload.commit_inputs(cols, log_rows, 16)` (blowup 4, 16 folds) through one
commit plan `repeat` times and prints the LDE root and the wall time of each run.
"""
import argparse
import time

import numpy as np

from . import native
from . import workload as wl

AIRS = {"seeded_fib": wl.AIR_SEEDED_FIB, "rescue_stacked": wl.AIR_RESCUE_STACKED, "ml_linear": wl.AIR_ML_LINEAR}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--air", choices=sorted(AIRS), default="rescue_stacked")
    ap.add_argument("--log-rows", type=int, default=18)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--sumcheck", choices=["gf8", "gf128"], default=None)
    ap.add_argument("--commit-cols", type=int, default=0, help="commit this many seeded columns instead of proving")
    args = ap.parse_args(argv)
    if args.commit_cols:
        trace, gammas, alphas = wl.commit_inputs(args.commit_cols, args.log_rows, 16)
        plan = native.CommitPlan(args.commit_cols, args.log_rows, 2, 16)
        plan.set_challenges(gammas, alphas)
        plan.upload(trace)
        for i in range(args.repeat):
            t0 = time.perf_counter()
            plan.run()
            root = plan.results()["lde_root"]
            print(f"commit {i}: root {root.hex()} in {1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)
        plan.close()
        return
    if args.sumcheck:
        es = 1 if args.sumcheck == "gf8" else 16
        hook = native.binius_gf256_values if es == 1 else native.binius_gf128_values
        n = 1 << args.log_rows
        tables = np.random.default_rng(args.seed).bytes(3 * n * es)
        for i in range(args.repeat):
            t0 = time.perf_counter()
            vals = hook(tables, n, 3, bytes([1] + [0] * (es - 1) + [2] + [0] * (es - 1)), [0, 1, 2, 0], [0, 3, 4], 3,
                        n // 2)
            print(f"round {i}: {vals.hex()} in {1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)
        return
    air, params, pi, trace, sep, pre = wl.proof_job(AIRS[args.air], args.log_rows, args.seed, b"zig-stark:cli")
    for i in range(args.repeat):
        t0 = time.perf_counter()
        proof = native.prove(air, params, pi, trace, pre, sep)
        print(f"proof {i}: {len(proof)} bytes in {1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)


if __name__ == "__main__":
    main()
