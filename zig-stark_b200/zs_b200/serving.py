"""Request streams over the proof server (zs_m31_server_*): open-loop arrivals,
continuous batching on the device, per-request latency.

A request is a tuple (air_id, params, public_inputs, trace, channel_sep[,
preprocessed]) of wire bytes (workload.ProofJob). `replay` submits each request at its arrival time from one thread while
another collects the results, so arrivals never wait for completions (open loop).
"""
import threading
import time

import numpy as np

from . import native


def poisson_arrivals(rate, duration, seed):
    """Arrival times (seconds from 0) of a Poisson process of `rate` per second over
    `duration` seconds, from a seeded generator."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)


def percentile(values, q):
    if not values:
        return float("nan")
    return float(np.percentile(np.asarray(values, dtype=np.float64), q))


def replay(requests, arrivals, workers, hbm_budget=0, keep_proofs=False):
    """Submits requests[i] at arrivals[i] to a fresh server with `workers` workers.

    Returns {"latency_ms": [...], "wall_s": first arrival to last completion,
    "completed": n, "failed": n, "proofs": [...] (when keep_proofs)}. Latency is the
    server's own submit-to-done time of each request."""
    assert len(requests) == len(arrivals)
    n = len(requests)
    tickets = [None] * n
    ready = [threading.Event() for _ in range(n)]
    lat = [None] * n
    proofs = [None] * n
    t_done = [0.0] * n
    with native.Server(workers=workers, hbm_budget=hbm_budget) as srv:
        t0 = time.perf_counter()

        def submitter():
            for i, (req, at) in enumerate(zip(requests, arrivals)):
                delay = t0 + at - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                air, params, pi, trace, sep = req[:5]
                pre = req[5] if len(req) > 5 else b""
                tickets[i] = srv.submit(air, params, pi, trace, pre, sep)
                ready[i].set()

        th = threading.Thread(target=submitter)
        th.start()
        for i in range(n):
            ready[i].wait()
            proof, ms = srv.poll(tickets[i], wait=True)
            t_done[i] = time.perf_counter()
            lat[i] = ms
            proofs[i] = proof if (keep_proofs or not isinstance(proof, bytes)) else b""
        th.join()
    failed = sum(1 for p in proofs if not isinstance(p, bytes))
    out = {"latency_ms": lat, "wall_s": (max(t_done) - (t0 + arrivals[0])) if n else 0.0,
           "completed": n - failed, "failed": failed}
    if keep_proofs:
        out["proofs"] = proofs
    return out
