"""Served process-map queries: a request loop with continuous batching.

Requests (directional-solidification solves) arrive as a Poisson stream. Each is initialised on a
host worker as soon as it arrives, admitted into the device pool as soon as it is initialised and
its HBM footprint fits the budget, stepped together with every other resident domain, and retired
(result copied out, memory freed) when it has met the reference's termination test. The results
of the domains that ended in one stretch of cycles are copied out while the next stretch runs (a
separate copy stream), and admission and retirement queue behind running cycles, so the device
steps while the host does its part. A domain's result does not depend on the others in the pool,
so each result equals its own plain run.
"""
from __future__ import annotations

import os
import queue
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import ExacaError, Pool
from .batch import build_problems, process_map


def request_stream(n_requests: int = 200, rate: float = 200.0, seed: int = 4, side=(48, 256), **map_kwargs) -> list:
    """Seeded Poisson arrivals (mean `rate` per second): [(arrival_s, params)], params as in
    batch.process_map with sides drawn from `side`."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    params = process_map(n_requests, seed=seed + 1000, side=side, **map_kwargs)
    return list(zip(arrivals.tolist(), params))


def serve(requests: list, device: int = 0, budget_bytes: int = 150 * 10**9, chunk_cycles: int = 250,
          list_capacity: int = 1 << 27, init_threads: int | None = None, keep_results: bool = False,
          deadline_s: float | None = None, pool_factory=Pool) -> dict:
    """Runs the request loop in real time and returns per-request latencies (s, arrival to result
    on the host), completion order and, with keep_results, each GrainID / CellType / final cycle
    (keep_results True: every request's; a set of request indices: those requests' only).

    deadline_s: a request whose result is not on the host that many seconds after its arrival is
    given up (its slot retired while the others run on, or never admitted); it is listed in
    `timed_out` and has no latency. pool_factory(device, budget_bytes=, list_capacity=) makes the
    pool (exaca_b200.Pool; tests pass a host-only stand-in)."""
    init_threads = init_threads or os.cpu_count() or 1
    n = len(requests)
    ready: queue.Queue = queue.Queue()
    t_start = time.perf_counter()

    def init_one(k):
        arrival, prm = requests[k]
        delay = t_start + arrival - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        try:
            prob = build_problems([prm], threads=1)[0]
            ready.put((k, prob, None))
        except Exception as e:  # reported through the loop
            ready.put((k, None, e))

    workers = ThreadPoolExecutor(max_workers=init_threads)
    for k in range(n):
        workers.submit(init_one, k)

    pool = pool_factory(device, budget_bytes=budget_bytes, list_capacity=list_capacity)
    latency = [None] * n
    results = [None] * n
    waiting = []  # initialised, not admitted yet (arrival order)
    resident = {}  # slot -> request index
    finished = []  # (slot, request index, final cycle) ended at the last status read
    timed_out = []
    done_count = 0
    steps = 0
    try:
        while done_count < n:
            # collect initialised requests
            try:
                while True:
                    k, prob, err = ready.get_nowait()
                    if err is not None:
                        raise err
                    waiting.append((k, prob))
            except queue.Empty:
                pass
            waiting.sort(key=lambda kp: requests[kp[0]][0])
            if deadline_s is not None:
                # give up requests past their deadline: waiting ones are dropped, resident ones
                # retired (those already ended on the device complete below)
                now = time.perf_counter() - t_start
                late = [kp for kp in waiting if now - requests[kp[0]][0] > deadline_s]
                waiting = [kp for kp in waiting if now - requests[kp[0]][0] <= deadline_s]
                for slot in [sl for sl, k in resident.items() if now - requests[k][0] > deadline_s]:
                    pool.retire(slot)
                    late.append((resident.pop(slot), None))
                for k, _ in late:
                    timed_out.append(k)
                    done_count += 1
            # admit in arrival order while the budget allows
            still = []
            for k, prob in waiting:
                if pool.bytes_in_use() + prob.slot_bytes() <= budget_bytes:
                    try:
                        slot = pool.admit(prob, device_check=True)
                        resident[slot] = k
                        continue
                    except ExacaError as e:
                        if e.code != -4:  # anything but a budget refusal is an error
                            raise
                still.append((k, prob))
            waiting = still
            if not resident and not finished:
                time.sleep(0.0005)
                continue
            if resident:
                pool.step(chunk_cycles)  # returns at launch
                steps += 1
            # results of the domains that ended before this stretch, while it runs
            for slot, k, cycle in finished:
                g, c = pool.copy_out_concurrent(slot)
                pool.retire(slot)
                latency[k] = time.perf_counter() - t_start - requests[k][0]
                if keep_results is True or (keep_results and k in keep_results):
                    results[k] = (g, c, cycle)
                done_count += 1
            finished = []
            if resident:
                slots = list(resident)
                for slot, st in zip(slots, pool.status_many(slots)):
                    if st.error:
                        raise ExacaError(-3, f"device error flags {st.error} in slot {slot}")
                    if st.done:
                        finished.append((slot, resident.pop(slot), st.cycle))
        elapsed = time.perf_counter() - t_start
    finally:
        workers.shutdown(wait=True)
        pool.close()
    lat = np.array([x for x in latency if x is not None], dtype=np.float64)
    return dict(latency=latency, results=results, elapsed=elapsed, solves_per_s=len(lat) / elapsed, steps=steps,
                timed_out=sorted(timed_out),
                p50=float(np.percentile(lat, 50)) if len(lat) else float("nan"),
                p99=float(np.percentile(lat, 99)) if len(lat) else float("nan"))


def sequential_plain(requests: list, device: int = 0) -> dict:
    """Sequential plain launches of the same requests: initialise, upload, run the reference's layer
    loop, copy out, one request after the other (arrival times ignored: the queue is always full)."""
    probs_needed = [prm for _, prm in requests]
    t0 = time.perf_counter()
    secs, results = [], []
    pool = None
    try:
        for prm in probs_needed:
            t = time.perf_counter()
            prob = build_problems([prm], threads=1)[0]
            if pool is None or prob.geometry.active_size > pool_cap:
                if pool is not None:
                    pool.close()
                pool_cap = max(prob.geometry.active_size, 1 << 20)
                pool = Pool(device, list_capacity=pool_cap)
            s = pool.admit(prob, device_check=False)
            cyc = pool.run_plain(s)
            g, c = pool.copy_out(s)
            pool.retire(s)
            results.append((g, c, cyc))
            secs.append(time.perf_counter() - t)
    finally:
        if pool is not None:
            pool.close()
    return dict(seconds=secs, results=results, elapsed=time.perf_counter() - t0,
                solves_per_s=len(secs) / (time.perf_counter() - t0))
