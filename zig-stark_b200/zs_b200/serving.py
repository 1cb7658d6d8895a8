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


def replay(requests, arrivals, workers, hbm_budget=0, keep_proofs=False, submitters=4):
    """Submits requests[i] at arrivals[i] to a fresh server with `workers` workers.

    `submitters` host threads share the submissions (request i goes to thread
    i % submitters), so a slow submit -- the server copies each request's buffers, which
    for a 200 MB trace takes tens of milliseconds -- does not hold back the arrivals
    behind it. Returns {"latency_ms": [...], "wall_s": first arrival to last
    completion, "completed": n, "failed": n, "submit_lag_ms": [...], "proofs": [...]
    (when keep_proofs)}. Latency is the server's own time from the start of a request's
    submit to its completion; submit_lag_ms is how late each submit started against its
    scheduled arrival."""
    assert len(requests) == len(arrivals)
    n = len(requests)
    tickets = [None] * n
    ready = [threading.Event() for _ in range(n)]
    lat = [None] * n
    lag = [0.0] * n
    proofs = [None] * n
    t_done = [0.0] * n
    k = max(1, min(submitters, n))
    with native.Server(workers=workers, hbm_budget=hbm_budget) as srv:
        t0 = time.perf_counter()

        def submitter(first):
            for i in range(first, n, k):
                req, at = requests[i], arrivals[i]
                delay = t0 + at - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                lag[i] = max(0.0, time.perf_counter() - (t0 + at)) * 1e3
                air, params, pi, trace, sep = req[:5]
                pre = req[5] if len(req) > 5 else b""
                tickets[i] = srv.submit(air, params, pi, trace, pre, sep)
                ready[i].set()

        ths = [threading.Thread(target=submitter, args=(f,)) for f in range(k)]
        for th in ths:
            th.start()
        for i in range(n):
            ready[i].wait()
            proof, ms = srv.poll(tickets[i], wait=True)
            t_done[i] = time.perf_counter()
            lat[i] = ms
            proofs[i] = proof if (keep_proofs or not isinstance(proof, bytes)) else b""
        for th in ths:
            th.join()
    failed = sum(1 for p in proofs if not isinstance(p, bytes))
    out = {"latency_ms": lat, "wall_s": (max(t_done) - (t0 + arrivals[0])) if n else 0.0,
           "completed": n - failed, "failed": failed, "submit_lag_ms": lag}
    if keep_proofs:
        out["proofs"] = proofs
    return out
