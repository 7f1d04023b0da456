"""Request-stream driver for the continuous-batching server (sdft_server_*).

Requests arrive at given times (a Poisson stream for the serving benchmark);
between launches the driver hands every arrived request to the server, runs
one server step (one kernel launch advancing every active request by a
bounded number of Anderson iterations) and collects the completions.  A
request's latency is the time from its arrival to the end of the step in
which it converged, including whatever the backend's submit and poll do at
arrival and completion (building the request, reading its result).

The backend is any object with submit(request, tag), step(iters) ->
(active, queued) and poll() -> [(tag, status, iters, err, device_ms)];
native.Server is the device one.
"""
from __future__ import annotations

import time

import numpy as np


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times (s) of n requests with exponential gaps at `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def serve_stream(backend, requests, arrivals, iters_per_step: int, clock=time.perf_counter, sleep=time.sleep):
    """Run the stream to completion; returns per-request results and summary statistics."""
    n = len(requests)
    arrivals = np.asarray(arrivals, dtype=np.float64)
    order = np.argsort(arrivals, kind="stable")
    done_at = np.full(n, np.nan)
    status = np.zeros(n, dtype=np.int32)
    iters = np.zeros(n, dtype=np.int32)
    errs = np.zeros(n)
    dev_ms = np.zeros(n)
    t0 = clock()
    nxt = 0
    finished = 0
    steps = 0
    active = queued = 0
    while finished < n:
        now = clock() - t0
        while nxt < n and arrivals[order[nxt]] <= now:
            i = int(order[nxt])
            backend.submit(requests[i], i)
            nxt += 1
            queued += 1
        if active == 0 and queued == 0:
            if nxt < n:  # idle until the next arrival
                sleep(max(0.0, arrivals[order[nxt]] - (clock() - t0)))
            continue
        active, queued = backend.step(iters_per_step)
        steps += 1
        t_end = clock() - t0
        for tag, st, it, err, dms in backend.poll():
            done_at[tag] = t_end
            status[tag] = st
            iters[tag] = it
            errs[tag] = err
            dev_ms[tag] = dms
            finished += 1
    wall = clock() - t0
    lat_ms = (done_at - arrivals) * 1e3
    return {
        "n": n,
        "steps": steps,
        "wall_s": wall,
        "solves_per_s": n / wall if wall > 0 else float("inf"),
        "p50_ms": float(np.percentile(lat_ms, 50)),
        "p99_ms": float(np.percentile(lat_ms, 99)),
        "latency_ms": lat_ms,
        "status": status,
        "iters": iters,
        "err": errs,
        "device_ms": dev_ms,
    }
