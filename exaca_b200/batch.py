"""Batched process maps: many directional-solidification domains of uneven sizes and parameters,
advanced together in one pool (one persistent kernel per stretch of cycles over the shared active
list), against the plain one-solve-at-a-time path.

The reference solves one domain per run (src/runCA.cpp:19-461); a process map is a loop over runs.
Here every domain is admitted into one pool with device-side termination, so each cycle's launch
advances all unfinished domains, and each domain's result is the one its own plain run gives
(the passes never mix domains: claims, captures and counters are per domain).
"""
from __future__ import annotations

import math
import os
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import INCONEL625, Pool, Problem


def process_map(n_domains: int = 256, seed: int = 3, side=(32, 128), G=(1e5, 5e6), R=(1e4, 1e6),
                density=(1e12, 1e15), dTN: float = 5.0, dTsigma: float = 0.5, fract_surface_active: float = 0.08,
                n_ratio: int = 25) -> list[dict]:
    """Seeded parameter sets of directional-solidification domains: each side uniform in `side`
    (cells, drawn per axis), G (K/m), R (K/s) and the bulk nucleation density (m^-3) log-uniform in
    their ranges; Inconel625 interfacial response, nucleation undercooling N(dTN, dTsigma)."""
    rng = np.random.default_rng(seed)

    def log_uniform(lo, hi):
        return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))

    out = []
    for _ in range(n_domains):
        nx, ny, nz = (int(v) for v in rng.integers(side[0], side[1] + 1, size=3))
        out.append(dict(nx=nx, ny=ny, nz=nz, G=log_uniform(*G), R=log_uniform(*R),
                        nucleation_density=log_uniform(*density) / 1e12, dTN=dTN, dTsigma=dTsigma,
                        fract_surface_active=fract_surface_active, n_ratio=n_ratio))
    return out


def footprint(p: dict) -> int:
    """Device bytes of a domain of these parameters (cells including the wall ring x the per-cell
    fields of a pool slot); the ranking that partitions a map over GPUs."""
    return (p["nx"] + 2) * (p["ny"] + 2) * (p["nz"] + 2) * 146


def partition(weights: list[int], n_parts: int) -> list[list[int]]:
    """Greedy bin-packing: items in decreasing weight, each to the currently lightest part (ties to
    the lowest part index). Deterministic, so every rank computes the same split without talking."""
    parts = [[] for _ in range(n_parts)]
    load = [0] * n_parts
    for i in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        j = min(range(n_parts), key=lambda q: (load[q], q))
        parts[j].append(i)
        load[j] += weights[i]
    return [sorted(p) for p in parts]


def build_problems(params: list[dict], threads: int | None = None) -> list[Problem]:
    """Host initialisation of every domain (independent, so it runs on a thread pool)."""
    threads = threads or os.cpu_count() or 1

    def one(p):
        return Problem.directional(p["nx"], p["ny"], p["nz"], G=p["G"], R=p["R"], n_ratio=p["n_ratio"],
                                   nucleation_density=p["nucleation_density"], dTN=p["dTN"], dTsigma=p["dTsigma"],
                                   fract_surface_active=p["fract_surface_active"], material=INCONEL625)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(one, params))


def solve_batch(problems: list[Problem], device: int = 0, autotune_cycles: int = 0, config: int | None = None,
                chunk_cycles: int = 1000) -> dict:
    """Admits every problem into one pool and steps them together until all have terminated.
    Returns per-domain GrainID / CellType / final cycle and the timings (s): admission (host->device),
    solve (device), copy-out (device->host)."""
    cap = sum(p.geometry.active_size for p in problems)
    pool = Pool(device, list_capacity=cap)
    try:
        t0 = time.perf_counter()
        slots = [pool.admit(p, device_check=True) for p in problems]
        t1 = time.perf_counter()
        tuned = None
        if config is not None:
            pool.set_config(config)
        if autotune_cycles:
            tuned = pool.autotune(autotune_cycles)
        pool.run_all(chunk_cycles)
        t2 = time.perf_counter()
        gids, cts, cycles = [], [], []
        for s in slots:
            g, c = pool.copy_out(s)
            gids.append(g)
            cts.append(c)
            cycles.append(pool.status(s).cycle)
        t3 = time.perf_counter()
        return dict(grain_id=gids, cell_type=cts, cycle=cycles, tuned=tuned,
                    seconds=dict(admit=t1 - t0, solve=t2 - t1, copy_out=t3 - t2, total=t3 - t0))
    finally:
        pool.close()


def solve_plain(problems: list[Problem], device: int = 0) -> dict:
    """The plain path: one domain at a time, each run as the reference's layer loop."""
    cap = max(p.geometry.active_size for p in problems)
    pool = Pool(device, list_capacity=cap)
    try:
        gids, cts, cycles, secs = [], [], [], []
        for p in problems:
            t0 = time.perf_counter()
            s = pool.admit(p, device_check=False)
            cycles.append(pool.run_plain(s))
            g, c = pool.copy_out(s)
            pool.retire(s)
            secs.append(time.perf_counter() - t0)
            gids.append(g)
            cts.append(c)
        return dict(grain_id=gids, cell_type=cts, cycle=cycles, seconds=secs)
    finally:
        pool.close()
