#!/usr/bin/env python
"""Benchmark of the B200 ExaCA solver on the 512^3 directional-solidification case.

Workload (one "step" = one complete solve, initial state -> termination): problem type C,
512 x 512 x 512 cells of 1 um (516 x 516 x 514 allocated with the wall ring), G = 1e6 K/m,
R = 1e6 K/s, N = 25 (dt = 0.04 us), Inconel625 interfacial response, 2 % of the bottom surface
seeded, bulk nucleation density 1e14 m^-3 with undercooling N(3 K, 0.5 K). Synthetic inputs: the
problem is generated from those parameters by the solver's own initialisation (seeded exactly as
the reference seeds it).

metric: cell-updates/s = active-window cells x CA cycles executed / solve time (the reference's
per-cycle sweep size times cycles). `value` is timed with CUDA events around each solve with the
initial state already resident in HBM; `e2e` times the same K solves through the C ABI, each
with its admission (upload of the seeds the cell fields are made from on the device, the fields'
construction), the solve and the GrainID/CellType download into pinned host buffers;
`e2e.with_host_init` adds the host's parsing and initialisation of the input file to every step, as
the drop-in executable runs it. The state (~20 GB) is larger than L2 and is rebuilt between steps.

`parity` checks the timed solve itself: SHA-256 digests of the last e2e solve's GrainID and CellType
against those pinned in tests/golden/DirS512.json (the oracle's restatement run to termination), and
of a solve stopped after cycle 5000 against the unmodified reference at that cycle. `batch` and
`serve` carry the process-map workloads (256 uneven domains in one pool; a Poisson request stream
with continuous batching) against their plain one-solve-per-launch paths, measured in the same run
(`--no-process-map` leaves them out; `--workload batch|serve` prints either alone).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--size S]
                    [--cpu-ref auto|reference|port]

`--impl reference` and the `cpu_baseline` time the reference's own OpenMP CPU path (built from its
sources against single-rank shims into oracle/_ref) on bounded samples of the same workload; when
that build is absent they time the oracle's serial restatement (oracle/_port) instead and say so
(`cpu_baseline.kind` "port").

For N > 1 (torchrun) every rank solves its own replica (the plain path has no exchange step) and
rank 0 prints the aggregate over ranks with the max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
UNIT = "cell-updates/s"
WORKLOAD = dict(G=1e6, R=1e6, n_ratio=25, nucleation_density=100.0, dTN=3.0, dTsigma=0.5, fract_surface_active=0.02)
REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
PORT_LIB = os.path.join(ROOT, "oracle", "_port", "liboracle.so")

# Algorithmic bytes of each pass per unit of work (the bytes the pass must read or write, each
# counted once per use, no cache reuse credited):
#   grow/claim: record 16 + domain 4 + liquid mask 4 + growth-table entry 8 per listed record;
#               diagonal/min-length write 8 per grown record; tombstone 16 + DiagonalLength 4 per
#               dropped record; critical-length row 104 + min write 4 per flagged record; 26
#               neighbour types + mask write 4 per fresh mask; 8 per claim + its TemporaryUpdate
#               CellType byte 1; 8 per listed target
#   capture:    per capture: claim 8, target 8, GrainID 4+4, centres 12+12, orientation 36,
#               DiagonalLength 4, 26 critical lengths 104, mask 4, record 16+4, CellType 1,
#               CritTimeStep 4, and per neighbour direction CellType 1 + two mask atomics 8; per
#               solidifying re-check CellType 1 + mask 4 (the mask word says whether it was grown)
PASS_BYTES = {
    "grow": dict(listed=24, grown=8, dropped=20, flagged=20),
    "claim": dict(flagged=20 + 104 + 4, fresh=30, claims=8 + 1 + 8),
    "capture": dict(claims=8 + 8, captured=221 + 26 * 9, rechecks=5),
}


def input_file_text(n):
    return "\n".join([
        f"Directional solidification {n}^3 (benchmark workload)",
        "*****",
        "Problem type: C",
        "Decomposition strategy: 1",
        "Material: Inconel625",
        "Cell size (microns): 1",
        "Heterogeneous nucleation density (normalized by 1*10^12 per m^3): 100",
        "Mean nucleation undercooling (in K): 3",
        "Standard deviation of nucleation undercooling: 0.5",
        "Path to output: ./",
        "Output file base name: bench",
        "File of grain orientations: GrainOrientationVectors_Uniform10k.csv",
        "Thermal gradient (K/m): 1000000",
        "Cooling rate (K/s): 1000000",
        f"Domain size in x: {n}",
        f"Domain size in y: {n}",
        f"Domain size in z: {n}",
        '"N", where the time step = deltax/(Steady State Velocity * N): 25',
        "Fraction of surface sites active: 0.02",
        "***Output data printing options: (Y or N) which data should be printed***",
        "Print Paraview vtk file of grain misorientation values (Y or N)?: N",
        "Print Paraview vtk file of all ExaCA data for post-processing (Y or N)?: N",
        "Debug check (reduced)- Print data for main Kokkos views (CellType, LayerID, CritTimeStep) following initialization for debug check (Y or N)?: N",
        "Debug check (extensive) - Print data for all main data structures (CellType, GrainID, CritTimeStep, UndercoolingCurrent, UndercoolingChange, Melted, LayerID) following initialization for debug check (Y or N)?: N",
    ]) + "\n"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def pinned_digests(n):
    """SHA-256 digests of the n^3 solve pinned in tests/golden/DirS<n>.json (GrainID as int32 and
    CellType as int8 over the whole cell array): at termination from the oracle's restatement, and
    after 5000 cycles from the reference itself. None when no such file was generated."""
    path = os.path.join(ROOT, "tests", "golden", f"DirS{n}.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def digests(grain_id, cell_type):
    import hashlib

    import numpy as np

    return {"sha_grain_id": hashlib.sha256(np.ascontiguousarray(grain_id, dtype=np.int32).tobytes()).hexdigest(),
            "sha_cell_type": hashlib.sha256(np.ascontiguousarray(cell_type).astype(np.int8).tobytes()).hexdigest()}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference_sample(n, samples, cycles_per_sample, threads):
    """The reference's own CPU path (OpenMP build) on bounded samples of the workload."""
    if not os.path.exists(REF_BENCH):
        raise FileNotFoundError(REF_BENCH)
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "bench.txt")
        with open(inp, "w") as f:
            f.write(input_file_text(n))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close",
                   EXACA_DATA_DIR=os.path.join(ROOT, "exaca_b200", "data"))
        r = subprocess.run([REF_BENCH, inp, str(samples), str(cycles_per_sample)], cwd=d, env=env,
                           capture_output=True, text=True, check=True)
        line = [ln for ln in r.stdout.splitlines() if "{\"cycles\"" in ln][-1]
        return json.loads(line[line.index("{"):])


def run_port_sample(n, samples, cycles_per_sample):
    """The oracle's serial restatement of the reference (one core) on bounded samples of the
    workload: the CPU baseline when the reference's own timing driver was not built."""
    import ctypes

    if not os.path.exists(PORT_LIB):
        raise FileNotFoundError(PORT_LIB)
    lib = ctypes.CDLL(PORT_LIB)
    lib.oracle_create.restype = ctypes.c_void_p
    lib.oracle_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    lib.oracle_error.restype = ctypes.c_char_p
    lib.oracle_geometry.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
    lib.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.oracle_free.argtypes = [ctypes.c_void_p]
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "bench.txt")
        with open(inp, "w") as f:
            f.write(input_file_text(n))
        t0 = time.perf_counter()
        o = lib.oracle_create(inp.encode(), os.path.join(ROOT, "exaca_b200", "data").encode())
        init_s = time.perf_counter() - t0
        if not o:
            raise RuntimeError(lib.oracle_error().decode())
        try:
            geo = (ctypes.c_longlong * 6)()
            lib.oracle_geometry(o, geo)
            times = []
            for _ in range(samples):
                t = time.perf_counter()
                lib.oracle_step(o, cycles_per_sample)
                times.append(time.perf_counter() - t)
        finally:
            lib.oracle_free(o)
    return {"sample_s": times, "active_domain_cells": int(geo[5]), "cycles_per_sample": cycles_per_sample,
            "cycles": samples * cycles_per_sample, "threads": 1, "init_s": init_s, "kind": "port"}


def cpu_sample(kind, n, samples, cycles_per_sample, threads):
    """Bounded samples of the reference's CPU path: its own OpenMP build when present ("reference"),
    else the oracle's serial restatement ("port")."""
    if kind == "reference" or (kind == "auto" and os.path.exists(REF_BENCH)):
        res = run_reference_sample(n, samples, cycles_per_sample, threads)
        res["kind"] = "reference"
        return res
    return run_port_sample(n, samples, cycles_per_sample)


def reference_arm(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    res = cpu_sample(args.cpu_ref, args.size, args.warmup + args.steps, args.ref_cycles, threads)
    timed = res["sample_s"][args.warmup:]
    cells = res["active_domain_cells"]
    cycles = res["cycles_per_sample"] * len(timed)
    value = cells * cycles / sum(timed)
    n = args.size
    path = ("the reference's OpenMP CPU path" if res["kind"] == "reference"
            else "the oracle's serial restatement of the reference")
    init = "the reference's own initialisation" if res["kind"] == "reference" else "the restatement's initialisation"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(timed) / len(timed), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32 (reference mixed precision)", "data": "synthetic",
        "config": {"workload": f"directional solidification {n}^3, G=R=1e6, N=25, 1e14 m^-3 nuclei",
                   "cells": cells, "step": f"{args.ref_cycles} CA cycles of {path}", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["threads"], "kind": res["kind"],
                         "sample": f"CA cycles {args.warmup * args.ref_cycles + 1}-{res['cycles']} of the {n}^3 "
                                   f"solve after {init} ({res['init_s']:.1f} s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def b200_arm(args, rank, world, local):
    import numpy as np
    import torch

    import exaca_b200 as ex

    if not os.path.exists(ex.LIB_PATH):
        from exaca_b200 import build as b

        b.build()
    device = local
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", device))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.size
    t0 = time.perf_counter()
    prob = ex.Problem.directional(n, n, n, **WORKLOAD)
    prob.pin()
    init_s = time.perf_counter() - t0
    g = prob.geometry
    cells = g.active_size
    pool = ex.Pool(device, list_capacity=cells)

    def solve():
        slot = pool.admit(prob, device_check=False)
        cyc = pool.run_plain(slot)
        ms = pool.last_run_ms()
        pool.retire(slot)
        return cyc, ms

    for _ in range(args.warmup):
        solve()
    barrier()
    st0 = pool.stats()
    clocks = ClockSampler(device)
    clocks.start()
    times, cycles = [], []
    for _ in range(args.steps):
        c, ms = solve()
        times.append(ms)
        cycles.append(c)
    clock_info = clocks.stop()
    barrier()
    st1 = pool.stats()
    total_ms = max_over_ranks(sum(times))
    cell_updates = cells * sum(cycles)
    value = world * cell_updates / (total_ms / 1e3)
    launches = st1["launches"] - st0["launches"] + sum(c // 1000 + 1 for c in cycles)  # + one census per 1000 cycles

    # end to end through the C ABI from pinned host buffers: upload, solve, download GrainID/CellType
    gid = torch.empty(g.domain_size, dtype=torch.int32, pin_memory=True)
    ct = torch.empty(g.domain_size, dtype=torch.int32, pin_memory=True)
    lib = ex.load_library()
    barrier()
    se0 = pool.stats()
    e2e_s, c_e = 0.0, 0
    for _ in range(args.steps):  # every step: admit (upload), solve, copy out; retirement untimed
        t_e = time.perf_counter()
        slot = pool.admit(prob, device_check=False)
        c_e += pool.run_plain(slot)
        rc = lib.exaca_pool_copy_out(pool._h, slot, gid.data_ptr(), ct.data_ptr())
        e2e_s += time.perf_counter() - t_e
        if rc != 0:
            raise RuntimeError(lib.exaca_last_error())
        pool.retire(slot)
    e2e_s = max_over_ranks(e2e_s)
    se1 = pool.stats()
    # the bytes the pool copied per step: the substrate seeds, plane CritTimeSteps and nuclei the
    # cell fields are made from on the device, the growth tables as the solve lengthens, GrainID and
    # CellType back
    h2d = (se1["h2d_bytes"] - se0["h2d_bytes"]) // args.steps
    d2h = (se1["d2h_bytes"] - se0["d2h_bytes"]) // args.steps
    e2e_value = world * cells * c_e / e2e_s

    # parity of the timed solve (untimed): the last e2e step's GrainID / CellType against the pinned
    # digests of the same input, and a second solve stopped after the reference-pinned cycle
    pins = pinned_digests(n)
    parity = {"checked": False, "why": f"no tests/golden/DirS{n}.json for this size"}
    if pins is not None:
        last = digests(gid.numpy(), ct.numpy())
        fin = pins.get("final", {})
        slot = pool.admit(prob, device_check=False)
        pool.step(pins["pin_cycle"])
        g5, c5 = pool.copy_out(slot)
        pool.retire(slot)
        at_pin = digests(g5, c5)
        del g5, c5
        ref_pin = pins.get("cycle5000_reference", {})
        parity = {
            "checked": True,
            "final_vs_restatement": bool(fin) and last == {k: fin[k] for k in last} and c_e == fin["cycle"] * args.steps,
            "final_cycle": c_e // args.steps, "restatement_final_cycle": fin.get("cycle"),
            f"cycle{pins['pin_cycle']}_vs_reference": bool(ref_pin) and at_pin == {k: ref_pin[k] for k in at_pin},
            "what": "SHA-256 of GrainID (int32) and CellType (int8) over all cells of the last e2e solve, against "
                    "the oracle's restatement run to termination; a further solve stopped after cycle "
                    f"{pins['pin_cycle']}, against the unmodified reference (Serial order) at that cycle "
                    "(tests/golden/make_dirs512.py)",
        }
        parity["ok"] = parity["final_vs_restatement"] and parity[f"cycle{pins['pin_cycle']}_vs_reference"]

    # end to end as the drop-in runs it: the input file parsed and the problem initialised on the
    # host (the reference's init), then admission, solve and copy-out, every step
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "bench.txt")
        with open(inp, "w") as f:
            f.write(input_file_text(n))
        barrier()
        full_s, c_f, init_f = 0.0, 0, 0.0
        host_steps = min(args.steps, 3)  # ~1.3 s of host initialisation each at 512^3
        for _ in range(host_steps):
            t_f = time.perf_counter()
            p_f = ex.Problem.from_file(inp)
            init_f += time.perf_counter() - t_f
            slot = pool.admit(p_f, device_check=False)
            c_f += pool.run_plain(slot)
            rc = lib.exaca_pool_copy_out(pool._h, slot, gid.data_ptr(), ct.data_ptr())
            full_s += time.perf_counter() - t_f
            if rc != 0:
                raise RuntimeError(lib.exaca_last_error())
            pool.retire(slot)
            del p_f
        full_s = max_over_ranks(full_s)

    # roofline of the persistent kernel (k_cycles, the only kernel of the timed solve apart from
    # the 1000-cycle census) on a bounded stretch of the solve: one launch, CUDA events around it
    slot = pool.admit(prob, device_check=False)
    pool.step(args.profile_at)
    pa = pool.stats()
    launch_ms = pool.timed_step(args.profile_cycles)
    pb = pool.stats()
    passes = pool.profile_cycles(args.profile_cycles)  # the same pass work as separate kernels
    pool.retire(slot)
    d = {k: pb[k] - pa[k] for k in pb}
    pass_bytes = {k: sum(per * d[unit] for unit, per in model.items()) for k, model in PASS_BYTES.items()}
    launch_bytes = sum(pass_bytes.values())
    peak, peak_kind = peaks()
    achieved = launch_bytes / (launch_ms / 1e3) / 1e9
    # ncu DRAM bytes per cycle of k_cycles, per cube side it was captured at ("k_cycles <side> <bytes>")
    traffic = None
    traffic_file = os.path.join(ROOT, "profiles", "traffic_per_launch.txt")
    if os.path.exists(traffic_file):
        for ln in open(traffic_file):
            f = ln.split()
            if len(f) == 3 and f[0] == "k_cycles" and int(f[1]) == n:
                traffic = float(f[2]) * args.profile_cycles

    # dense-equivalent effective roofline (the reference formulation's compulsory bytes per cycle)
    eff_bytes_per_update = 14.5

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32 (reference mixed precision), int32/int8",
            "data": "synthetic (generated by the solver's own seeded initialisation)",
            "config": {"workload": f"directional solidification {n}^3, G=R=1e6 K/m|K/s, N=25, 1e14 m^-3 nuclei",
                       "cells": cells, "cycles": cycles, "step": "one full solve to termination",
                       "l2": "state (~148 B/cell, > L2) re-uploaded between steps", "replicas": world,
                       "host_init_s": round(init_s, 2)},
            "clocks": clock_info,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "seconds": e2e_s,
                    "with_host_init": {"value": world * cells * c_f / full_s, "unit": UNIT, "seconds": full_s,
                                       "steps": host_steps, "host_init_s_per_step": init_f / host_steps,
                                       "what": "input file parsed and problem initialised on the host every "
                                               "step, then admission, solve and copy-out"}},
            "parity": parity,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "k_cycles", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": "not measured in this run: ncu DRAM bytes per cycle of a 1000-cycle "
                                           "k_cycles launch (profiles/traffic_per_launch.txt) x the cycles of "
                                           "this launch; the 512^3 figure is from an earlier kernel version "
                                           "(the current one moves 32 % fewer DRAM bytes per cycle at 288^3, "
                                           "profiles/k_cycles_dirsolid288_dram.md)",
                         "algorithmic_bytes_per_launch": launch_bytes, "launch_ms": launch_ms,
                         "sample": f"one launch over cycles {args.profile_at + 1}-{args.profile_at + args.profile_cycles}",
                         "pass_bytes_per_launch": pass_bytes,
                         "separate_pass_ms_per_cycle": {k: v / max(1, args.profile_cycles) for k, v in passes.items()},
                         "effective_dense_frac": value / world * eff_bytes_per_update / 1e9 / peak},
        }
        if world == 1 and not args.no_cpu_baseline:
            try:
                # the reference arm's cycle window at the same --steps / --warmup: `warmup` untimed samples
                # of ref_cycles cycles after initialisation, then `steps` timed ones
                threads = os.cpu_count() or 1
                res = cpu_sample(args.cpu_ref, n, args.warmup + args.steps, args.ref_cycles, threads)
                timed = res["sample_s"][args.warmup:]
                v = res["active_domain_cells"] * res["cycles_per_sample"] * len(timed) / sum(timed)
                what = ("reference OpenMP CPU path after its own initialisation" if res["kind"] == "reference"
                        else "oracle's serial restatement of the reference")
                first = args.warmup * args.ref_cycles + 1
                line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": res["threads"], "kind": res["kind"],
                                        "sample": f"CA cycles {first}-{res['cycles']} of the same {n}^3 solve "
                                                  f"(cycles 1-{first - 1} untimed), {what}"}
            except Exception as e:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                                        "sample": f"unavailable: {e}"}
    pool.close()
    # the process-map workloads (batched and served solves/s against their plain paths) under the
    # same clock, as objects of the same line
    if not args.no_process_map:
        b = measure_batch(args, rank, world, local, dist, 1, 1)
        sv = measure_serve(args, rank, world, local, dist, 1, 1)
        if rank == 0:
            line["batch"] = b
            line["serve"] = sv
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _dist_setup(world, local):
    """NCCL process group for the multi-GPU workloads (barrier and max over ranks only)."""
    import datetime

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
        return dist
    return None


def _max_over_ranks(dist, x):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measure_batch(args, rank, world, local, dist, steps, warmup):
    """Batched process map (256 uneven directional domains, every domain bit-exact with its own plain
    run): batched solves/s against the plain one-domain-at-a-time path on a seeded sample. Host
    initialisation is excluded from both arms (every problem is built before either clock starts).
    With N GPUs the map is split by HBM footprint (greedy bin-packing, no per-cycle exchange) and
    the time is the slowest rank's. Returns the measurement on rank 0, None elsewhere."""
    import numpy as np

    from exaca_b200 import batch

    all_params = batch.process_map(args.domains, seed=3)
    mine = batch.partition([batch.footprint(p) for p in all_params], world)[rank]
    params = [all_params[i] for i in mine]
    t0 = time.perf_counter()
    probs = batch.build_problems(params)
    init_s = time.perf_counter() - t0
    for _ in range(warmup):
        batch.solve_batch(probs[:8], device=local, config=0)
    times, tuned, res = [], None, None
    for _ in range(steps):
        if dist is not None:
            dist.barrier()
        res = batch.solve_batch(probs, device=local, autotune_cycles=50)
        times.append(_max_over_ranks(dist, res["seconds"]["total"]))
        tuned = res["tuned"]
    exact, plain, sample = None, None, []
    if rank == 0:
        rng = np.random.default_rng(7)
        sample = sorted(rng.choice(len(probs), size=min(args.plain_sample, len(probs)), replace=False).tolist())
        pl = batch.solve_plain([probs[i] for i in sample], device=local)
        exact = all(pl["cycle"][j] == res["cycle"][i] and np.array_equal(pl["grain_id"][j], res["grain_id"][i])
                    and np.array_equal(pl["cell_type"][j], res["cell_type"][i]) for j, i in enumerate(sample))
        plain = len(sample) / sum(pl["seconds"])
    if dist is not None:
        dist.barrier()
    if rank != 0:
        return None
    value = len(all_params) / min(times)
    return {
        "metric": "batched solves/s", "value": value, "unit": "solves/s", "steps": steps, "warmup": warmup,
        "ms_per_step": 1e3 * min(times), "scaling": "strong",
        "workload": f"batched process map, {len(all_params)} directional domains, sides 32-128 per axis, "
                    "G 1e5-5e6 K/m, R 1e4-1e6 K/s, nucleation 1e12-1e15 m^-3 (log-uniform)",
        "rank0_cells": int(sum(p.geometry.active_size for p in probs)), "rank0_host_init_s": round(init_s, 2),
        "parallelism": f"{world} GPU(s), domains split by footprint",
        "step": "admit all, autotune, step until every domain terminated, copy out all",
        "host_init": "excluded from both arms",
        "plain_solves_per_s": plain, "speedup_vs_plain": value / plain,
        "plain_sample": f"{len(sample)} seeded domains of rank 0 solved one at a time on one GPU (admit, run, copy out)",
        "sample_bit_exact": bool(exact), "autotune": {"config": tuned[0], "ms_per_cycle": tuned[1]},
        "cycles": {"max": int(max(res["cycle"])), "median": float(np.median(res["cycle"]))},
        "seconds": res["seconds"],
    }


def measure_serve(args, rank, world, local, dist, steps, warmup):
    """Served process-map queries: Poisson arrivals (200/s) admitted under a 150 GB HBM budget per
    GPU and stepped together; solves/s and p50/p99 latency against sequential plain launches of the
    first requests. Host initialisation is included in both arms (a served request is initialised
    when it arrives; a plain launch initialises, admits, runs and copies out). The plain sample's
    results must equal the served ones. With N GPUs requests are routed by footprint (greedy
    bin-packing of the stream, no per-cycle exchange); solves/s uses the slowest rank's wall time,
    latency percentiles all requests. Returns the measurement on rank 0, None elsewhere."""
    import numpy as np

    from exaca_b200 import batch, serve

    all_reqs = serve.request_stream(args.requests, rate=200.0, seed=4)
    mine = batch.partition([batch.footprint(p) for _, p in all_reqs], world)[rank]
    reqs = [all_reqs[i] for i in mine]
    n_plain = min(args.plain_sample, len(reqs))
    for w in range(warmup):
        serve.serve(serve.request_stream(8, rate=200.0, seed=100 + w, side=(24, 48)), device=local)
    runs = []
    for _ in range(steps):
        if dist is not None:
            dist.barrier()
        runs.append(serve.serve(reqs, device=local, keep_results=set(range(n_plain)) if rank == 0 else False))
    best = max(runs, key=lambda r: r["solves_per_s"])
    elapsed = _max_over_ranks(dist, best["elapsed"])
    lat = [x for x in best["latency"] if x is not None]
    if dist is not None:
        gathered = [None] * world
        dist.all_gather_object(gathered, lat)
        lat = [x for part in gathered for x in part]
    pl, exact = None, None
    if rank == 0:
        pl = serve.sequential_plain(reqs[:n_plain], device=local)
        exact = all(r is not None and q[2] == r[2] and np.array_equal(q[0], r[0]) and np.array_equal(q[1], r[1])
                    for q, r in zip(pl["results"], best["results"][:n_plain]))
    if dist is not None:
        dist.barrier()
    if rank != 0:
        return None
    value = len(all_reqs) / elapsed
    return {
        "metric": "served solves/s", "value": value, "unit": "solves/s", "steps": steps, "warmup": warmup,
        "ms_per_step": 1e3 * elapsed, "scaling": "strong",
        "workload": f"served process-map queries, {len(all_reqs)} requests, Poisson 200/s, sides 48-256 per axis, "
                    "G/R/nucleation as the batched map, 150 GB HBM budget per GPU",
        "parallelism": f"{world} GPU(s), requests routed by footprint",
        "step": "real-time request loop until every request's result is on the host",
        "host_init": "included in both arms",
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "timed_out": len(best["timed_out"]),
        "plain_solves_per_s": pl["solves_per_s"], "speedup_vs_plain": value / pl["solves_per_s"],
        "plain_sample": f"first {len(pl['seconds'])} requests of rank 0 launched one after the other on one GPU "
                        "(init, admit, run, copy out)",
        "sample_bit_exact": bool(exact),
    }


def workload_arm(args, rank, world, local):
    """`--workload batch|serve`: one JSON line for the process-map workload alone."""
    dist = _dist_setup(world, local)
    measure = measure_batch if args.workload == "batch" else measure_serve
    m = measure(args, rank, world, local, dist, args.steps, args.warmup)
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": m.pop("metric"), "value": m.pop("value"), "unit": m.pop("unit"), "n_gpus": world,
        "steps": m.pop("steps"), "warmup": m.pop("warmup"), "ms_per_step": m.pop("ms_per_step"),
        "higher_is_better": True, "scaling": m.pop("scaling"), "vs_baseline": None,
        "dtype": "f64/f32 (reference mixed precision), int32/int8",
        "data": "synthetic (seeded process map)" if args.workload == "batch" else
                "synthetic (seeded Poisson request stream)",
        "config": {"workload": m.pop("workload"), "parallelism": m.pop("parallelism"), "step": m.pop("step")},
    }
    line.update(m)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--ref-cycles", type=int, default=20, help="CA cycles per reference sample")
    ap.add_argument("--profile-at", type=int, default=6000)
    ap.add_argument("--profile-cycles", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-process-map", action="store_true",
                    help="plain workload without the batched / served process-map objects")
    ap.add_argument("--cpu-ref", default="auto", choices=["auto", "reference", "port"],
                    help="CPU path timed by --impl reference and the cpu_baseline: the reference's own OpenMP "
                         "build (oracle/_ref), the oracle's serial restatement, or the former when built")
    ap.add_argument("--workload", default="plain", choices=["plain", "batch", "serve"],
                    help="plain: the 512^3 headline; batch / serve: the process-map workloads (1 GPU)")
    ap.add_argument("--domains", type=int, default=256)
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--plain-sample", type=int, default=32)
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        reference_arm(args, rank, world)
    elif args.workload in ("batch", "serve"):
        workload_arm(args, rank, world, local)
    else:
        b200_arm(args, rank, world, local)


if __name__ == "__main__":
    main()
