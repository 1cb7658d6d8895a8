"""Command line: prove synthetic traces on the GPU (for timing and profiling runs).

    PYTHONPATH=zig-stark_b200 python -m zs_b200.cli --air rescue_stacked --log-rows 18 --repeat 2

proves the same job `repeat` times through zs_m31_prove and prints the proof size and
the wall time of each call. The job is `workload.proof_job(air, log_rows, seed, sep)`:
blowup 4, 16 queries, remainder_log 3.
"""
import argparse
import time

from . import native
from . import workload as wl

AIRS = {"seeded_fib": wl.AIR_SEEDED_FIB, "rescue_stacked": wl.AIR_RESCUE_STACKED, "ml_linear": wl.AIR_ML_LINEAR}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--air", choices=sorted(AIRS), default="rescue_stacked")
    ap.add_argument("--log-rows", type=int, default=18)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--seed", type=int, default=3)
    args = ap.parse_args(argv)
    air, params, pi, trace, sep, pre = wl.proof_job(AIRS[args.air], args.log_rows, args.seed, b"zig-stark:cli")
    for i in range(args.repeat):
        t0 = time.perf_counter()
        proof = native.prove(air, params, pi, trace, pre, sep)
        print(f"proof {i}: {len(proof)} bytes in {1e3 * (time.perf_counter() - t0):.2f} ms", flush=True)


if __name__ == "__main__":
    main()
