"""Benchmark of the circle commit workload on B200.

Workload (one step): 64 columns x 2^20 rows of uniform M31 values; circle IFFT on the
canonic 2^20 domain, circle FFT on the canonic 2^22 domain (blowup 4), Blake3 row
leaves (hashM31s of each 64-value row) and the full Merkle tree, the QM31 combination
g = sum_c gamma_c * LDE_c, then 16 FRI folds 2^22 -> 2^6 with seeded challenges, each
layer committed (hashQM31 leaves + tree) before it is folded.

Metric: trace rows per second of the whole step (value = 2^20 * n_gpus / step time).
Inputs (256 MiB trace, 1 GiB LDE) are larger than the 126 MB L2, so no flush is needed
between steps. `e2e` times the same step through the C ABI with the host trace copied
from pinned memory every step and the roots / final layer read back, with two steps in
flight (two commit plans on two streams, so one step's upload overlaps the other's
compute); `pipelined` also gives the device time with two steps in flight, and
`e2e.one_at_a_time_ms_per_step` the end-to-end time of one step at a time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "zig-stark_b200"))

N_COLS, LOG_ROWS, LOG_BLOWUP, N_FOLDS = 64, 20, 2, 16
METRIC = "M31 LDE+Merkle commit rows/s (64 cols x 2^20, blowup 4, + 16-fold FRI chain)"
UNIT = "rows/s"
# The oracle's LDE root of the timed workload (oracle.circle_commit on
# workload.commit_inputs(64, 20, 16), blowup 4), so the timed configuration is checked
# against the oracle without running it at full size on every bench.
ORACLE_LDE_ROOT = {20: "0482a2ea4854035e11838b72cc7360faaacf1779a8d52908dd28ccba2b1cb397"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--log-rows", type=int, default=LOG_ROWS, help="smaller cases for profiling")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-binius", action="store_true", help="skip the Binius sum-check figures")
    ap.add_argument("--no-pipeline", action="store_true", help="skip the two-steps-in-flight figures")
    ap.add_argument("--no-proofs", action="store_true",
                    help="skip the proof workloads and the reference-kernel bar after the commit step")
    ap.add_argument("--workload", default="commit", choices=["commit", "prove", "batch", "serve"],
                    help="commit: the circle commit step (default); prove: single proofs (Fibonacci 2^12, "
                         "stacked Rescue 2^18); batch: mixed-size proof batch, batched vs one at a time; "
                         "serve: Poisson request stream, p50/p99 latency")
    ap.add_argument("--jobs", type=int, default=512, help="batch: number of traces")
    ap.add_argument("--batch-arm", default="both", choices=["both", "plain"],
                    help="batch: 'plain' runs only the one-at-a-time arm and reports each shape's time "
                         "(for profiling the proofs one by one)")
    ap.add_argument("--log-min", type=int, default=None)
    ap.add_argument("--log-max", type=int, default=None)
    ap.add_argument("--concurrency", type=int, default=8, help="batch / serve: prover workers")
    ap.add_argument("--rate", type=float, default=400.0, help="serve: arrivals per second")
    ap.add_argument("--duration", type=float, default=5.0, help="serve: seconds of arrivals")
    return ap.parse_args()


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons while the timed region runs:
    through NVML every 10 ms (read-only queries, the GPU found by its UUID), else
    nvidia-smi every 200 ms."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []  # (sm_mhz, max_mhz, [active reason names])
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            try:
                h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(torch.cuda.get_device_properties(device).uuid))
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self._nvml = (pynvml, h)
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        nv, h = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.rows.append((float(sm), float(mx), [n for n, m in self.REASONS if bits & m]))

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=5).stdout.strip()
        r = [x.strip() for x in out.split(",")] if out else []
        if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
            self.rows.append((float(r[1]), float(r[2]),
                              [n for i, (n, _) in enumerate(self.REASONS) if r[5 + i] == "Active"]))

    def _run(self):
        period = 0.01 if self._nvml else 0.2
        while True:
            try:
                self._sample_nvml() if self._nvml else self._sample_smi()
            except Exception:
                pass
            if self._stop.wait(period):
                break

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(r[0] for r in self.rows)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted({n for r in self.rows for n in r[2]}), "samples": len(self.rows),
                "source": "nvml" if self._nvml else "nvidia-smi"}


def dist_setup(args, backend="nccl"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)  # each rank's NCCL communicator on its own GPU
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world):
    """Max of a per-rank float over all ranks (the slowest replica sets the step time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline_sample(threads):
    """The oracle restatement on a bounded sample of the workload: all 64 columns at
    2^16 rows, blowup 4, 10 folds, with the reference's per-call twiddle recomputation."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from zs_b200 import workload as wl
    log_rows, folds = 16, 10
    trace, gammas, alphas = wl.commit_inputs(N_COLS, log_rows, folds)
    oracle.circle_commit(trace[:, :1 << 10][:8], LOG_BLOWUP, gammas[:8], alphas[:4], faithful=True, threads=threads)
    t0 = time.perf_counter()
    oracle.circle_commit(trace, LOG_BLOWUP, gammas, alphas, faithful=True, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": (1 << log_rows) / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"64 cols x 2^{log_rows} rows, blowup 4, {folds} folds (per-call twiddles as the "
                      f"reference computes them), {dt:.2f} s"}


def commit_config(log_rows, world):
    """The commit workload's `config`, shared by both arms of the benchmark."""
    return {"workload": "circle commit: 64 cols x 2^20 M31, blowup 4, row-leaf Blake3 Merkle, "
                        "16-fold QM31 FRI chain with per-layer commits",
            "columns": N_COLS, "log_rows": log_rows, "log_blowup": LOG_BLOWUP, "folds": N_FOLDS,
            "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (no flush)"}


def run_reference(args, world, rank):
    """The reference's CPU path (restated: Zig is not available) on the host cores, on
    this benchmark's config and metric: each step times a bounded sample of the
    workload (64 columns x 2^16 rows, 10 folds; about a second on 16 cores), and rows/s
    of the sample stand for the full 2^20-row commit's (per row, the sample's transforms
    are a little shorter, so the CPU figure errs high)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    samples = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline_sample(threads)
        if i >= args.warmup:
            samples.append(cb["value"])
    v = sum(samples) / len(samples)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (1 << 16) / v * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31)", "data": "synthetic",
            "impl": "reference",
            "config": commit_config(LOG_ROWS, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": cb["sample"] + "; rank 0 alone under torchrun"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# proof workloads: a mixed-size batch, and a served request stream
# ---------------------------------------------------------------------------

def _proof_jobs(shapes, cache_variants=None):
    """Wire-format jobs for (air, log_rows, seed, sep) shapes. With cache_variants,
    traces repeat per (air, log_rows) across that many seeds (each request keeps its
    own channel separator, so every proof differs)."""
    from zs_b200 import workload as wl
    cache, jobs = {}, []
    for i, (air, lg, seed, sep) in enumerate(shapes):
        key = (air, lg, i % cache_variants) if cache_variants else i
        if key not in cache:
            cache[key] = wl.proof_job(air, lg, seed, sep)
        jobs.append(cache[key]._replace(sep=sep))
    return jobs


def _cpu_prove_sample(jobs, max_log, count):
    """The oracle prover (NTT route, OpenMP over the host cores) on the first `count`
    jobs with at most 2^max_log rows."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    pick = [j for j in jobs if j[1][0] <= max_log][:count]
    t0 = time.perf_counter()
    for air, params, pi, trace, sep, pre in pick:
        oracle.prove(air, params, pi, pre, trace, sep, mode=1)
    dt = time.perf_counter() - t0
    return {"value": len(pick) / dt, "unit": "proofs/s", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": f"{len(pick)} jobs of the stream with <= 2^{max_log} rows, oracle NTT prover, {dt:.2f} s"}


def run_prove(args, world, rank, local):
    """Single proofs through zs_m31_prove from host buffers, one at a time: the
    2^12-row Fibonacci AIR (a_1 seeded, blowup 4, 16 queries, separator
    "zig-stark:fibonacci:example"), stacked Rescue at 2^18 rows and the linear layer
    (W 128 x 128, 2^14 input vectors, 2^15 rows), all at blowup 4."""
    import torch
    from zs_b200 import native, wire
    from zs_b200 import workload as wl
    torch.cuda.set_device(local)
    fib_tr, fib_pi = wl.seeded_fib(12)
    fib = wl.ProofJob(wl.AIR_SEEDED_FIB, wire.StarkParams(12, 2, 16, 3).encode(), fib_pi, wire.columns(fib_tr),
                      b"zig-stark:fibonacci:example", b"")
    cases = {"seeded_fib_2^12": fib,
             "rescue_stacked_2^18": wl.proof_job(wl.AIR_RESCUE_STACKED, 18, wl.SEED_RESCUE, b"zig-stark:rescue:stacked"),
             "ml_linear_2^14_vectors": wl.proof_job(wl.AIR_ML_LINEAR, 15, wl.SEED_ML_LINEAR,
                                                    b"zig-stark:ml_linear:layer")}
    out = {}
    with ClockSampler(local) as clocks:
        for name, (air, params, pi, trace, sep, pre) in cases.items():
            proof = None
            for _ in range(args.warmup):
                proof = native.prove(air, params, pi, trace, pre, sep)
            barrier(world)
            ts = []
            for _ in range(args.steps):
                t0 = time.perf_counter()
                p = native.prove(air, params, pi, trace, pre, sep)
                ts.append(time.perf_counter() - t0)
            assert p == proof, "proof changed between runs"
            ms = max_over_ranks(sorted(ts)[len(ts) // 2], world) * 1e3
            out[name] = {"ms_per_proof_median": ms, "ms_min": min(ts) * 1e3, "proofs_per_s": world * 1e3 / ms,
                         "proof_bytes": len(proof), "trace_bytes": len(trace)}
    line = {
        "metric": "single-proof latency through zs_m31_prove (host buffers in, proof bytes out)",
        "value": out["rescue_stacked_2^18"]["proofs_per_s"], "unit": "proofs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": out["rescue_stacked_2^18"]["ms_per_proof_median"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31 / QM31 exact)", "data": "synthetic (seeded)",
        "config": {"workload": "stacked Rescue 2^18 rows (value); SeededFib 2^12 rows and the linear layer "
                               "(W 128 x 128, 2^14 input vectors) also timed; blowup 4, 16 queries",
                   "parallelism": f"replicas x{world}"},
        "cases": out,
        "e2e": {"value": out["rescue_stacked_2^18"]["proofs_per_s"], "unit": "proofs/s",
                "h2d_bytes_per_step": out["rescue_stacked_2^18"]["trace_bytes"],
                "d2h_bytes_per_step": out["rescue_stacked_2^18"]["proof_bytes"]},
        "roofline": None, "gpu_launches": None, "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        air, params, pi, trace, sep, _ = fib
        t0 = time.perf_counter()
        want = oracle.prove(air, params, pi, b"", trace, sep, mode=1)
        dt = time.perf_counter() - t0
        got = native.prove(air, params, pi, trace, b"", sep)
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "proofs/s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"SeededFib 2^12 proof by the oracle (NTT route), {dt * 1e3:.1f} ms"}
        line["parity"] = {"seeded_fib_2^12_bytes_equal_oracle": got == want}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batch(args, world, rank, local):
    """Independent traces (Fibonacci / stacked Rescue 50/50 by seed, log2 rows uniform
    in 10..20, blowup 4, 16 queries, a channel separator per trace), proven batched
    (zs_m31_prove_batch) and one at a time (zs_m31_prove), both from host buffers."""
    import torch
    from zs_b200 import native
    from zs_b200 import workload as wl
    torch.cuda.set_device(local)
    lo, hi = args.log_min or 10, args.log_max or 20
    shapes = wl.batch_shapes(args.jobs, log_min=lo, log_max=hi)[rank::world]
    jobs = _proof_jobs(shapes)
    kw = [dict(air_id=a, params=p, public_inputs=pi, trace=t, preprocessed=pre, channel_sep=sp)
          for a, p, pi, t, sp, pre in jobs]
    h2d = sum(len(j[3]) + len(j[1]) + len(j[2]) for j in jobs)

    def batched():
        return native.prove_batch(kw, concurrency=args.concurrency)

    def plain():
        return [native.prove(**k) for k in kw]

    if args.batch_arm == "plain":
        ref = plain()
        per_shape = {}
        for _ in range(args.steps):
            for k, (air, params, *_rest) in zip(kw, jobs):
                t0 = time.perf_counter()
                native.prove(**k)
                per_shape.setdefault(f"{air}:{params[0]}", []).append(time.perf_counter() - t0)
        if rank == 0:
            print(json.dumps({"workload": "batch", "arm": "plain", "jobs": args.jobs, "steps": args.steps,
                              "plain_s_per_pass": sum(sum(v) for v in per_shape.values()) / args.steps,
                              "per_shape_ms": {k: {"count": len(v) // args.steps, "ms_median": 1e3 * sorted(v)[len(v) // 2]}
                                               for k, v in sorted(per_shape.items())}}), flush=True)
        return

    ref = batched()  # grows the device pool to the batch's working set
    assert all(isinstance(p, bytes) for p in ref), "a batch job failed"
    for _ in range(max(0, args.warmup - 1)):
        batched()
    d2h = sum(len(p) for p in ref)

    def timed(fn, k):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            out = fn()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        barrier(world)
        return max_over_ranks(dt, world) / k, out

    with ClockSampler(local) as clocks:
        t_b, got = timed(batched, args.steps)
    assert got == ref, "batched proofs changed between runs"
    plain()  # warm the one-at-a-time path
    t_p, got_p = timed(plain, args.steps)
    assert got_p == ref, "one-at-a-time proofs differ from the batched ones"
    value = args.jobs / t_b
    line = {
        "metric": "proofs/s, batched (mixed-size Fibonacci/Rescue stream)", "value": value,
        "unit": "proofs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_b * 1e3, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32 (M31 / QM31 exact)", "data": "synthetic (SplitMix64 seeded)",
        "config": {"workload": f"{args.jobs} traces, SeededFib / stacked Rescue 50/50 by seed, log2 rows "
                               f"uniform in {lo}..{hi}, blowup 4, 16 queries, per-trace channel separator",
                   "concurrency": args.concurrency, "parallelism": f"jobs sharded over {world} replica(s)",
                   "l2": "working set far above L2"},
        "plain_value": args.jobs / t_p, "plain_ms_per_step": t_p * 1e3,
        "batched_over_plain": t_p / t_b,
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "the prover API takes host buffers and returns host proofs: every step is end to end"},
        "roofline": None,
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _cpu_prove_sample(jobs, 13, 24)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_serve(args, world, rank, local):
    """Poisson arrivals at --rate per second for --duration seconds; each request a
    Fibonacci, stacked Rescue or linear-layer proof (50/30/20) with log2 rows from a
    geometric distribution (p = 0.5) truncated to 12..22 (the linear layer capped at
    2^15 rows). Served with continuous batching
    (--concurrency workers) and, on the same arrivals, one request at a time."""
    import torch
    from zs_b200 import serving
    from zs_b200 import workload as wl
    torch.cuda.set_device(local)
    lo, hi = args.log_min or 12, args.log_max or 22
    arrivals = serving.poisson_arrivals(args.rate, args.duration, wl.SEED_SERVE + rank)
    shapes = wl.serve_shapes(len(arrivals), seed=wl.SEED_SERVE + 7919 * rank, log_min=lo, log_max=hi)
    jobs = _proof_jobs(shapes, cache_variants=2)
    # warm-up: the largest shapes, so the device pool already holds the working set
    warm = sorted(set((j[0], j[1][0]) for j in jobs), key=lambda x: -x[1])[:4]
    wjobs = [next(j for j in jobs if (j[0], j[1][0]) == w) for w in warm]
    serving.replay(wjobs * 2, [0.0] * (2 * len(wjobs)), args.concurrency)
    barrier(world)
    with ClockSampler(local) as clocks:
        served = serving.replay(jobs, arrivals, args.concurrency)
    plain = serving.replay(jobs, arrivals, 1)
    barrier(world)
    wall = max_over_ranks(served["wall_s"], world)
    wall_p = max_over_ranks(plain["wall_s"], world)
    n_total = len(jobs) * world
    lat, lat_p = served["latency_ms"], plain["latency_ms"]
    line = {
        "metric": "proofs/s and p50/p99 latency, served stream (continuous batching)",
        "value": n_total / wall, "unit": "proofs/s", "n_gpus": world, "steps": 1, "warmup": 1,
        "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 (M31 / QM31 exact)", "data": "synthetic (SplitMix64 seeded; traces repeat over 2 seeds "
                                                   "per shape, every request has its own channel separator)",
        "config": {"workload": f"Poisson {args.rate:g} req/s for {args.duration:g} s per GPU, SeededFib / "
                               f"stacked Rescue / linear layer 50/30/20, log2 rows geometric(0.5) truncated "
                               f"to {lo}..{hi} (linear layer at most 2^15), "
                               "blowup 4, 16 queries", "requests": n_total, "concurrency": args.concurrency,
                   "parallelism": f"replicas x{world}"},
        "latency_ms": {"p50": serving.percentile(lat, 50), "p99": serving.percentile(lat, 99),
                       "max": max(lat) if lat else None},
        "plain": {"value": n_total / wall_p, "p50": serving.percentile(lat_p, 50),
                  "p99": serving.percentile(lat_p, 99)},
        "failed": served["failed"] + plain["failed"],
        "e2e": {"value": n_total / wall, "unit": "proofs/s",
                "h2d_bytes_per_step": sum(len(j[3]) for j in jobs), "d2h_bytes_per_step": None,
                "note": "requests arrive as host buffers and proofs return to the host"},
        "roofline": None, "gpu_launches": None, "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def proof_metrics(args, local, budget_s=90.0):
    """The proof configurations, bounded for the default run (about a minute), on one
    GPU: single-proof latency of the 2^12-row SeededFib proof (bytes checked against
    the oracle), of the 2^18-row stacked Rescue proof and of the linear layer (W 128 x
    128, 2^14 input vectors); the 512-trace mixed batch (SeededFib / stacked Rescue
    50/50, log2 rows 10..20), batched against one at a time; and the served stream
    (SeededFib / stacked Rescue / linear layer 50/30/20, log2 rows geometric over
    12..22) at three arrival rates, with p50/p99 latency, against one request at a time
    at the middle rate. Traces repeat per (AIR, size) over two seeds; every job has its
    own channel separator, so every proof differs."""
    import torch
    from zs_b200 import native, serving, wire
    from zs_b200 import workload as wl
    t_start = time.perf_counter()
    out = {}
    fib_tr, fib_pi = wl.seeded_fib(12)
    singles = {"seeded_fib_2^12": wl.ProofJob(wl.AIR_SEEDED_FIB, wire.StarkParams(12, 2, 16, 3).encode(), fib_pi,
                                              wire.columns(fib_tr), b"zig-stark:fibonacci:example", b""),
               "rescue_stacked_2^18": wl.proof_job(wl.AIR_RESCUE_STACKED, 18, wl.SEED_RESCUE,
                                                   b"zig-stark:rescue:stacked"),
               "ml_linear_2^14_vectors": wl.proof_job(wl.AIR_ML_LINEAR, 15, wl.SEED_ML_LINEAR,
                                                      b"zig-stark:ml_linear:layer")}
    for name, (air, params, pi, trace, sep, pre) in singles.items():
        proof = native.prove(air, params, pi, trace, pre, sep)
        for _ in range(3):
            native.prove(air, params, pi, trace, pre, sep)
        ts = []
        for _ in range(15):
            t0 = time.perf_counter()
            p = native.prove(air, params, pi, trace, pre, sep)
            ts.append(time.perf_counter() - t0)
        assert p == proof, "proof changed between runs"
        out[name] = {"ms_median": sorted(ts)[len(ts) // 2] * 1e3, "ms_min": min(ts) * 1e3,
                     "proof_bytes": len(proof), "trace_bytes": len(trace) + len(pre)}
        if name.startswith("seeded_fib"):
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            out[name]["bytes_equal_oracle"] = proof == oracle.prove(air, params, pi, pre, trace, sep, mode=1)
    # 512 mixed-size traces, batched vs one at a time
    jobs = _proof_jobs(wl.batch_shapes(512), cache_variants=2)
    kw = [dict(air_id=a, params=p, public_inputs=pi, trace=t, preprocessed=pre, channel_sep=sp)
          for a, p, pi, t, sp, pre in jobs]
    # 16 workers: batched throughput over 512 jobs rises from 4 to 16 workers (535, 570,
    # 596 proofs/s) and falls at 32 (583), the device being full
    ref = native.prove_batch(kw, concurrency=16)  # grows the device pool to the batch's working set
    assert all(isinstance(p, bytes) for p in ref), "a batch job failed"
    native.prove_batch(kw, concurrency=16)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(2):
        got = native.prove_batch(kw, concurrency=16)
    t_b = (time.perf_counter() - t0) / 2
    assert got == ref, "batched proofs changed between runs"
    t0 = time.perf_counter()
    got_p = [native.prove(**k) for k in kw]
    t_p = time.perf_counter() - t0
    assert got_p == ref, "one-at-a-time proofs differ from the batched ones"
    out["batch_512"] = {"batched_proofs_per_s": len(kw) / t_b, "plain_proofs_per_s": len(kw) / t_p,
                        "batched_over_plain": t_p / t_b, "batched_s": t_b, "plain_s": t_p,
                        "workload": "512 traces, SeededFib / stacked Rescue 50/50, log2 rows uniform 10..20, "
                                    "blowup 4, 16 queries, concurrency 16"}
    # served stream at three rates, and one at a time at the middle rate
    serve = {}
    for rate in (100.0, 400.0, 1200.0):
        if time.perf_counter() - t_start > budget_s:
            serve[f"{rate:g}"] = {"skipped": "time budget of the default run"}
            continue
        arrivals = serving.poisson_arrivals(rate, 4.0, wl.SEED_SERVE)
        sjobs = _proof_jobs(wl.serve_shapes(len(arrivals)), cache_variants=2)
        if rate == 100.0:  # warm the pool with the largest shapes
            warm = sorted(set((j[0], j[1][0]) for j in sjobs), key=lambda x: -x[1])[:4]
            wjobs = [next(j for j in sjobs if (j[0], j[1][0]) == w) for w in warm]
            serving.replay(wjobs * 2, [0.0] * (2 * len(wjobs)), 8)
        r = serving.replay(sjobs, arrivals, 8)
        lat = r["latency_ms"]
        row = {"requests": len(sjobs), "proofs_per_s": len(sjobs) / r["wall_s"],
               "p50_ms": serving.percentile(lat, 50), "p99_ms": serving.percentile(lat, 99), "failed": r["failed"],
               "submit_lag_p99_ms": serving.percentile(r["submit_lag_ms"], 99)}
        if rate == 400.0:
            rp = serving.replay(sjobs, arrivals, 1)
            row["plain"] = {"proofs_per_s": len(sjobs) / rp["wall_s"],
                            "p50_ms": serving.percentile(rp["latency_ms"], 50),
                            "p99_ms": serving.percentile(rp["latency_ms"], 99)}
        serve[f"{rate:g}"] = row
    out["serve"] = {"workload": "Poisson arrivals for 4 s per rate, SeededFib / stacked Rescue / linear layer "
                                "50/30/20, log2 rows geometric(0.5) truncated to 12..22 (linear layer capped at "
                                "2^15 rows), blowup 4, 16 queries, 8 workers",
                    "rates": serve}
    out["wall_s"] = time.perf_counter() - t_start
    return out


def reference_gpu_bar(n_cols=64):
    """The reference's own GPU circle FFT (its kernels built from its source for sm_100a,
    driven as src/cuda/circlefft_gpu.zig does: one launch per layer), timed on this
    GPU for the commit workload's transforms: the circleIFFT of 2^20 points and the
    circleFFT of 2^22 points per column. Device time of its launches per column (host
    twiddles by the coset walk, which gives the same values faster), scaled to the 64
    columns, and one whole reference call at 2^16 points with its per-call host twiddles."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref not built (the reference tree was absent at build time)"}
    from zs_b200 import workload as wl
    x20 = wl.uniform_m31(0x5EED00F0, 1 << 20)
    x22 = wl.uniform_m31(0x5EED00F1, 1 << 22)
    ref_gpu.set_fast_twiddles(True)
    for _ in range(2):
        ref_gpu.ifft(x20)
        ref_gpu.fft(x22)
    dev_i, dev_f = [], []
    for _ in range(3):
        dev_i.append(ref_gpu.ifft(x20)[2])
        dev_f.append(ref_gpu.fft(x22)[2])
    ref_gpu.set_fast_twiddles(False)
    x16 = wl.uniform_m31(0x5EED00F2, 1 << 16)
    ref_gpu.fft(x16)
    _, wall16, dev16 = ref_gpu.fft(x16)
    ref_gpu.set_fast_twiddles(True)
    di, df = min(dev_i), min(dev_f)
    return {"ifft_2^20_device_ms_per_column": di, "fft_2^22_device_ms_per_column": df,
            "lde_device_ms_64_columns": n_cols * (di + df),
            "fft_2^16_call_ms": wall16, "fft_2^16_call_device_ms": dev16,
            "note": "reference kernels src/cuda/kernels/circlefft.cu compiled for sm_100a, one launch per layer; "
                    "device ms are CUDA events around its launches; the call at 2^16 includes its host "
                    "twiddles, allocations and copies"}


SC_TERMS = [([0, 1, 2], 1), ([0], 2)]  # src/cuda/sumcheck_test.zig:40-43: t0 t1 t2 + 2 t0


def _sc_lookups_per_row(bits, terms, dmax):
    """GF(2^8) table lookups the round kernel makes per row for `terms` (its own
    arithmetic: a GF(2^128) product is 121 lookups, a subfield scalar times a GF(2^128)
    element 16, a GF(2^8) product 1; the points 0..3 need none for the linear factor,
    a unit coefficient none, a GF(2^8) coefficient of a GF(2^128) term 16)."""
    mul, scal = (1, 1) if bits == 8 else (121, 16)
    total = 0
    for fs, c in terms:
        if not fs:
            continue
        for t in range(dmax + 1):
            total += (scal if t >= 4 else 0) * len(fs) + mul * (len(fs) - 1)
            if c != 1:
                total += mul if (bits == 8 or c >= 256) else scal
    return total


def binius_metrics(clock_mhz):
    """The Binius sum-check (src/binius/sumcheck.zig; its GPU hook src/binius/accel.zig),
    three tables and the terms of src/cuda/sumcheck_test.zig, seeded random elements:
    one round's values on tables resident in device memory (a CUDA graph of 20 rounds,
    CUDA events), the hook with host tables (copies included), and the whole combination
    prover; beside the reference's own kernels (src/cuda/kernels/sumcheck.cu built for
    sm_100a, driven as src/cuda/sumcheck_gpu.zig does: copies per call, one thread per
    row) and the oracle's single-threaded CPU prover at a smaller size. The round kernel
    is bound by shared-memory table lookups: its roofline is lookups per second against
    one lookup per lane per cycle on every SM."""
    import numpy as np
    import torch
    from zs_b200 import native
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import ref_gpu
    idx, off = [0, 1, 2, 0], [0, 3, 4]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = {"terms": "t0 t1 t2 + 2 t0 over 3 tables (src/cuda/sumcheck_test.zig:40-43)", "dmax": 3}
    wavefronts = {8: 3.11, 128: 2.96}
    for bits, k, k_cpu in ((8, 24, 16), (128, 20, 10)):
        es = 1 if bits == 8 else 16
        n = 1 << k
        rng = np.random.default_rng(0x5EED0100 + bits)
        tables = rng.bytes(3 * n * es)
        coeffs = b"".join(c.to_bytes(es, "little") for _, c in SC_TERMS)
        hook = native.binius_gf256_values if bits == 8 else native.binius_gf128_values
        d_cur = torch.frombuffer(bytearray(tables), dtype=torch.uint8).cuda()
        d_out = torch.zeros(64, dtype=torch.uint8, device="cuda")
        s = torch.cuda.Stream()
        call = lambda: native.binius_values_device(bits, d_cur.data_ptr(), n, 3, SC_TERMS, 3, n // 2,  # noqa: E731
                                                   d_out.data_ptr(), s.cuda_stream)
        with torch.cuda.stream(s):
            call()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        reps = 20
        with torch.cuda.graph(g, stream=s):
            for _ in range(reps):
                call()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        for _ in range(3):
            g.replay()
        torch.cuda.synchronize()
        dev = []
        for _ in range(3):
            ev[0].record(s)
            with torch.cuda.stream(s):
                g.replay()
            ev[1].record(s)
            torch.cuda.synchronize()
            dev.append(ev[0].elapsed_time(ev[1]) / reps)
        dev_ms = min(dev)
        got = hook(tables, n, 3, coeffs, idx, off, 3, n // 2)
        hook_ms = []
        for _ in range(3):  # pageable host tables, as the reference's hook receives them
            t0 = time.perf_counter()
            hook(tables, n, 3, coeffs, idx, off, 3, n // 2)
            hook_ms.append((time.perf_counter() - t0) * 1e3)
        per_row = _sc_lookups_per_row(bits, SC_TERMS, 3)
        achieved = (n // 2) * per_row / (dev_ms * 1e-3)
        peak = sms * 32 * clock_mhz * 1e6
        r = {"rows": n, "round_device_ms": dev_ms, "round_rows_per_s": n / (dev_ms * 1e-3),
             "hook_ms": min(hook_ms), "hook_h2d_bytes": 3 * n * es,
             "roofline": {"bound": "shared-memory lookups", "lookups_per_row_pair": per_row,
                          "achieved": achieved, "peak": peak, "unit": "lookups/s", "frac": achieved / peak,
                          "peak_basis": f"{sms} SMs x 32 lanes x {clock_mhz:.0f} MHz",
                          # shared-memory wavefronts per warp lookup at random addresses,
                          # from an ncu capture of the round kernels at these sizes
                          "wavefronts_per_lookup": wavefronts[bits],
                          "frac_of_bank_conflict_ceiling": achieved / peak * wavefronts[bits]}}
        if ref_gpu.sumcheck_available():
            ref_gpu.sumcheck_values(bits == 128, tables, n, 3, coeffs, idx, off, 3, n // 2)
            runs = [ref_gpu.sumcheck_values(bits == 128, tables, n, 3, coeffs, idx, off, 3, n // 2) for _ in range(2)]
            r["reference_kernel_device_ms"] = min(x[2] for x in runs)
            r["reference_hook_ms"] = min(x[1] for x in runs)
            r["reference_values_equal"] = all(x[0] == got for x in runs)
            r["round_speedup_vs_reference_kernel"] = r["reference_kernel_device_ms"] / dev_ms
        else:
            r["reference_kernel"] = "unavailable: oracle/_ref not built (the reference tree was absent)"
        pinned = torch.frombuffer(bytearray(tables), dtype=torch.uint8).pin_memory()

        def best_ms(fn, reps=3):
            fn()
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                fn()
                ts.append((time.perf_counter() - t0) * 1e3)
            return min(ts)

        r["hook_pinned_ms"] = best_ms(lambda: hook(pinned, n, 3, coeffs, idx, off, 3, n // 2))
        # the whole proof from host tables: k rounds, every round's values and fold on the device
        r["prove_ms"] = best_ms(lambda: native.binius_prove_combination(bits, pinned, k, 3, SC_TERMS))
        r["prove_pageable_ms"] = best_ms(lambda: native.binius_prove_combination(bits, tables, k, 3, SC_TERMS))
        r["prove_input"] = "prove_ms: tables in pinned host memory; prove_pageable_ms: a Python bytes object"
        small = rng.bytes(3 * (1 << k_cpu) * es)
        t0 = time.perf_counter()
        want = oracle.binius_prove(7 if bits == 128 else 3, small, k_cpu, 3, SC_TERMS)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        mine = native.binius_prove_combination(bits, small, k_cpu, 3, SC_TERMS)
        r[f"prove_2^{k_cpu}_ms"] = (time.perf_counter() - t0) * 1e3
        r[f"cpu_oracle_prove_2^{k_cpu}_ms"] = cpu_ms
        r[f"prove_2^{k_cpu}_equal_oracle"] = mine == want
        out[f"gf2^{bits}"] = r
        del d_cur, g
    return out


def main():
    args = parse()
    # the reference arm runs on the host cores only: its ranks meet over gloo
    world, rank, local = dist_setup(args, backend="gloo" if args.impl == "reference" else "nccl")
    if args.impl == "reference":
        run_reference(args, world, rank)
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload in ("prove", "batch", "serve"):
        {"prove": run_prove, "batch": run_batch, "serve": run_serve}[args.workload](args, world, rank, local)
        barrier(world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import numpy as np
    import torch
    from zs_b200 import native
    from zs_b200 import workload as wl

    torch.cuda.set_device(local)
    log_rows = args.log_rows
    trace, gammas, alphas = wl.commit_inputs(N_COLS, log_rows, N_FOLDS)
    plan = native.CommitPlan(N_COLS, log_rows, LOG_BLOWUP, N_FOLDS)
    plan.set_challenges(gammas, alphas)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    pinned = torch.from_numpy(trace.view(np.int32)).pin_memory()
    plan.upload(pinned.data_ptr(), sp)
    torch.cuda.synchronize()

    # correctness of the timed configuration: the first run against the oracle's root
    plan.run(None, sp)
    ref_root = plan.results(sp)["lde_root"]
    root_ok = ref_root.hex() == ORACLE_LDE_ROOT[log_rows] if log_rows in ORACLE_LDE_ROOT else None

    def timed(fn, k):
        barrier(world)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(k):
            fn()
        end.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return start.elapsed_time(end)

    # device-resident step
    for _ in range(args.warmup):
        plan.run(None, sp)
    with ClockSampler(local) as clocks:
        ms = timed(lambda: plan.run(None, sp), args.steps)
    ms = max_over_ranks(ms, world)
    ms_step = ms / args.steps

    # per-phase breakdown with events on the launching stream
    phase_ms = {}
    for ph, name in enumerate(native.CommitPlan.PHASES):
        evs = []
        for _ in range(max(1, args.steps // 2)):
            for p2 in range(ph):
                plan.run_phase(p2, None, sp)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            plan.run_phase(ph, None, sp)
            b.record(stream)
            for p2 in range(ph + 1, 3):
                plan.run_phase(p2, None, sp)
            evs.append((a, b))
        torch.cuda.synchronize()
        phase_ms[name] = sum(a.elapsed_time(b) for a, b in evs) / len(evs)

    # end to end through the C ABI: H2D of the trace from pinned memory, run, read back
    h2d = trace.nbytes
    d2h = 32 + 32 * N_FOLDS + (1 << (log_rows + LOG_BLOWUP - N_FOLDS)) * 16
    e2e_s = float("nan")
    if not args.no_e2e:
        for _ in range(args.warmup):
            plan.run_host(pinned.data_ptr(), sp)
            plan.results(sp)
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            plan.run_host(pinned.data_ptr(), sp)  # the upload overlaps the LDE of earlier column groups
            r = plan.results(sp)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world) / args.steps
        assert r["lde_root"] == ref_root, "e2e run changed the LDE root"

    # two steps in flight: a second plan on a second stream, so one step's upload and LDE
    # overlap the other's row tree and folds (every step still does all its work: its
    # upload from pinned memory, its commit, its results read back)
    pipe = None
    if not args.no_pipeline:
        plan2 = native.CommitPlan(N_COLS, log_rows, LOG_BLOWUP, N_FOLDS)
        plan2.set_challenges(gammas, alphas)
        stream2 = torch.cuda.Stream()
        sp2 = stream2.cuda_stream
        plan2.upload(pinned.data_ptr(), sp2)
        plans, sps = (plan, plan2), (sp, sp2)

        def dev_pipe(k):
            for i in range(k):
                plans[i % 2].run(None, sps[i % 2])

        dev_pipe(max(2, args.warmup))
        barrier(world)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        stream2.wait_event(start)
        dev_pipe(args.steps)
        stream.wait_stream(stream2)
        end.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        pipe_ms = max_over_ranks(start.elapsed_time(end), world) / args.steps
        assert plan2.results(sp2)["lde_root"] == ref_root, "the second plan's LDE root differs"
        pipe_e2e_s = float("nan")
        if not args.no_e2e:
            for i in range(max(2, args.warmup)):
                plans[i % 2].run_host(pinned.data_ptr(), sps[i % 2])
            for i in range(2):
                plans[i].results(sps[i])
            barrier(world)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for i in range(args.steps):
                plans[i % 2].run_host(pinned.data_ptr(), sps[i % 2])
                if i > 0:  # the previous step's results, read while this step runs
                    r = plans[(i - 1) % 2].results(sps[(i - 1) % 2])
            r = plans[(args.steps - 1) % 2].results(sps[(args.steps - 1) % 2])
            pipe_e2e_s = max_over_ranks(time.perf_counter() - t0, world) / args.steps
            assert r["lde_root"] == ref_root, "pipelined e2e run changed the LDE root"
        plan2.close()
        rows_ = (1 << log_rows) * world
        pipe = {"steps_in_flight": 2, "ms_per_step": pipe_ms, "rows_per_s": rows_ / (pipe_ms / 1e3),
                "e2e_ms_per_step": pipe_e2e_s * 1e3, "e2e_rows_per_s": rows_ / pipe_e2e_s,
                "how": "two commit plans on two streams, steps alternating between them; device time "
                       "with CUDA events across both streams, end to end by the host clock with every "
                       "step's upload from pinned memory and its results read back"}

    rows = (1 << log_rows) * world
    value = rows / (ms_step / 1e3)
    # end to end: with two steps in flight when measured (each step's upload overlaps the
    # other's compute; the copy of 256 MiB bounds it), else one step at a time
    e2e_line = {"value": rows / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_s * 1e3, "steps_in_flight": 1}
    if pipe is not None and pipe["e2e_ms_per_step"] == pipe["e2e_ms_per_step"]:
        e2e_line.update({"value": pipe["e2e_rows_per_s"], "ms_per_step": pipe["e2e_ms_per_step"],
                         "steps_in_flight": 2, "one_at_a_time_ms_per_step": e2e_s * 1e3})
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    # dominant phase and its algorithmic bytes (inputs and outputs it must touch)
    n, N = 1 << log_rows, 1 << (log_rows + LOG_BLOWUP)
    alg = {
        "lde": N_COLS * (n + N) * 4,                      # read trace, write LDE
        "row_tree": N_COLS * N * 4 + (2 * N - 1) * 32 * 2 + N * 16,  # read LDE, write 2 trees + g
        "folds": sum((N >> i) * 16 + (N >> (i + 1)) * 16 + (2 * (N >> (i + 1)) - 1) * 32 for i in range(N_FOLDS)),
    }
    dom = max(phase_ms, key=phase_ms.get)
    achieved = alg[dom] / (phase_ms[dom] / 1e3) / 1e9
    # DRAM read + write bytes per launch of each phase's kernels from ncu, scaled by the
    # rows. LDE: its three kernels at 32 columns x 2^20 rows (1.945 GB; the intermediate
    # buffers are larger than L2 there too) scaled to 64 columns. Row leaves + trees: the
    # row leaves and the row and g trees of this workload (1381.5 MB read, 443.0 MB
    # written; one pass per launch, checked on the 32-column case first).
    traffic = {"lde": 1.9454e9 * (N_COLS / 32) * 2.0 ** (log_rows - 20),
               "row_tree": 1.8245e9 * 2.0 ** (log_rows - 20)}.get(dom)
    # Integer co-roof. The path is exact integer work, so next to the HBM roof each phase
    # is set against the SMs' issue rate (148 SMs x 4 schedulers x 1 warp instruction per
    # cycle at the sampled SM clock) and against the ALU pipe's (a warp instruction every
    # other cycle per scheduler), with the warp instructions that ncu counted for the
    # phase's kernels on this workload (smsp__inst_executed.sum and
    # sm__inst_executed_pipe_alu.sum of one captured step at 64 x 2^20, summed over each
    # phase's kernels), over the CUDA-event phase time of this run. Other row counts
    # scale the counts by the rows (marked).
    counted = {"lde": (946.8e6, 488.4e6), "row_tree": (1059.4e6, 735.3e6), "folds": (342.0e6, 237.1e6)}
    cs = clocks.summary()
    sm_mhz = cs.get("sm_mhz") or cs.get("sm_max_mhz") or 1965.0
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    issue_peak = n_sm * 4 * sm_mhz * 1e6  # warp instructions per second
    scale = 2.0 ** (log_rows - LOG_ROWS)
    int_roof = {"bound": "integer issue", "unit": "warp instructions/s", "issue_peak": issue_peak,
                "alu_pipe_peak": issue_peak / 2,
                "source": "ncu counters of this workload's kernels (smsp__inst_executed.sum, "
                          "sm__inst_executed_pipe_alu.sum) from one captured step at 64 x 2^20"
                          + ("" if log_rows == LOG_ROWS else f"; scaled by 2^{log_rows - LOG_ROWS} rows"),
                "phases": {}}
    for k, (inst, alu) in counted.items():
        sec = phase_ms[k] / 1e3
        int_roof["phases"][k] = {"warp_instructions": inst * scale, "alu_warp_instructions": alu * scale,
                                 "issue_frac": inst * scale / sec / issue_peak,
                                 "alu_pipe_frac": alu * scale / sec / (issue_peak / 2)}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (M31 / QM31 exact)", "data": "synthetic (SplitMix64 seeded)",
        "config": commit_config(log_rows, world),
        "phases_ms": phase_ms,
        "parity": {"lde_root_equal_oracle": root_ok},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "algorithmic_bytes": alg[dom]},
        "int_roofline": int_roof,
        "pipelined": pipe,
        "commit_bytes_per_row": 1536,
        "e2e": e2e_line,
        "gpu_launches": plan.launches() * args.steps,
        "clocks": cs,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and log_rows == LOG_ROWS:
        line["cpu_baseline"] = cpu_baseline_sample(os.cpu_count() or 1)
    plan.close()
    if world == 1 and log_rows == LOG_ROWS and not args.no_proofs:
        try:
            line["reference_gpu_circle_fft"] = reference_gpu_bar()
        except Exception as e:  # the bar is reported, never required
            line["reference_gpu_circle_fft"] = {"unavailable": f"{type(e).__name__}: {e}"}
        line["proofs"] = proof_metrics(args, local)
    if world == 1 and log_rows == LOG_ROWS and not args.no_binius:
        line["binius_sumcheck"] = binius_metrics(cs.get("sm_mhz") or 1965.0)
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
