"""B200-native ExaCA cellular-automaton solver: Python host-side interface.

The product is the native library ``lib/libexaca_b200.so`` (C++ host code + sm_100a CUDA kernels
behind the C ABI declared in ``include/exaca_b200.h``). This module binds that ABI with ctypes and
mirrors the reference's entry points:

* :func:`run_program` is ``RunProgram_Reduced(id, np, InputFile)`` (src/runCA.hpp:11) at one rank:
  input file in, ``.vtk`` / ``_Misorientations.vtk`` / ``.log`` out.
* :class:`Problem` is the reference's initialisation (src/CAinitialize.hpp:16-96).
* :class:`Pool` holds device-resident domains and advances them with the step kernels that replace
  ``Nucleation`` / ``CellCapture`` / ``IntermediateOutputAndCheck`` (src/CAupdate.hpp:15-33).

There is no CPU fallback: if the native library is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libexaca_b200.so")
EXE_PATH = os.path.join(_HERE, "lib", "ExaCA-B200")
DATA_DIR = os.path.join(_HERE, "data")

# CellType codes (src/CAtypes.hpp:11)
WALL, SOLID, ACTIVE, TEMPORARY_UPDATE, TEMPORARY_INIT, LIQUID, GHOST = range(7)
VORONOI_PENDING = -(2**31)

ERRORS = {
    -1: "input error",
    -2: "unsupported problem",
    -3: "CUDA error",
    -4: "admission refused",
    -5: "bad argument",
}


class ExacaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class ProblemGeometry(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("mx", ctypes.c_int), ("my", ctypes.c_int), ("nz_active", ctypes.c_int),
        ("domain_size", ctypes.c_int64), ("active_size", ctypes.c_int64),
        ("n_nuclei", ctypes.c_int), ("deltat", ctypes.c_double), ("simulation_type", ctypes.c_char),
    ]


class DirsParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("cell_size_um", ctypes.c_double), ("G", ctypes.c_double), ("R", ctypes.c_double),
        ("n_ratio", ctypes.c_int), ("nucleation_density", ctypes.c_double),
        ("dTN", ctypes.c_double), ("dTsigma", ctypes.c_double), ("fract_surface_active", ctypes.c_double),
        ("A", ctypes.c_double), ("B", ctypes.c_double), ("C", ctypes.c_double), ("D", ctypes.c_double),
        ("freezing_range", ctypes.c_double),
    ]


class DomainStatus(ctypes.Structure):
    _fields_ = [
        ("cycle", ctypes.c_int), ("done", ctypes.c_int), ("nn", ctypes.c_int), ("error", ctypes.c_int),
        ("liquid", ctypes.c_int64), ("layer", ctypes.c_int), ("window_z_lo", ctypes.c_int),
        ("window_nz", ctypes.c_int), ("reserved", ctypes.c_int),
    ]


class PoolStatsT(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("cycles", "launches", "listed", "grown", "captured", "nucleated", "claims", "row_reads", "dropped",
                 "fresh", "rechecks", "flagged", "h2d_bytes", "d2h_bytes")]


class CensusT(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("superheated", "undercooled", "active", "solid", "remaining", "next_cts")]


class CellFieldsT(ctypes.Structure):
    """exaca_cell_fields: device pointers to one domain's CellType / LayerID / CritTimeStep."""
    _fields_ = [
        ("cell_type", ctypes.c_void_p), ("layer_id", ctypes.c_void_p), ("crit_time_step", ctypes.c_void_p),
        ("domain_size", ctypes.c_int64), ("active_size", ctypes.c_int64), ("cycle", ctypes.c_int32),
        ("layer", ctypes.c_int32), ("window_start", ctypes.c_int64),
    ]


CENSUS_MAX_DOMAINS = 256
STEP_CONFIGS = 8
# device error flags (exaca_domain_status.error; include/exaca_b200.h EXACA_FLAG_*)
FLAG_GROWTH_TABLE, FLAG_LIST_OVERFLOW, FLAG_BOUNDS, FLAG_BARRIER = 1, 2, 4, 8

class GrainStatsT(ctypes.Structure):
    _fields_ = [("region_cells", ctypes.c_int64), ("melted_cells", ctypes.c_int64), ("n_grains", ctypes.c_int64),
                ("mean_grain_volume_um3", ctypes.c_double), ("nucleated_fraction", ctypes.c_double),
                ("mean_misorientation_deg", ctypes.c_double), ("mean_misorientation_top_deg", ctypes.c_double),
                ("misorientation_hist", ctypes.c_uint64 * 64)]


# Every symbol include/exaca_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_I = ctypes.c_int
SIGNATURES = {
    "exaca_last_error": ([], ctypes.c_char_p),
    "exaca_run_program": ([ctypes.c_char_p, _I], _I),
    "exaca_problem_from_file": ([ctypes.c_char_p, ctypes.POINTER(_P)], _I),
    "exaca_problem_directional": ([ctypes.POINTER(DirsParams), ctypes.POINTER(_P)], _I),
    "exaca_problem_free": ([_P], None),
    "exaca_problem_info": ([_P, ctypes.POINTER(ProblemGeometry)], _I),
    "exaca_problem_fields": ([_P, _P, _P, _P, _P, _P], _I),
    "exaca_problem_slot_bytes": ([_P], ctypes.c_int64),
    "exaca_pool_create": ([_I, ctypes.c_size_t, ctypes.c_uint64, ctypes.POINTER(_P)], _I),
    "exaca_pool_destroy": ([_P], None),
    "exaca_pool_admit": ([_P, _P, _I, ctypes.POINTER(_I)], _I),
    "exaca_pool_step": ([_P, _I], _I),
    "exaca_pool_status": ([_P, _I, ctypes.POINTER(DomainStatus)], _I),
    "exaca_pool_census": ([_P, _I, ctypes.POINTER(CensusT)], _I),
    "exaca_pool_stats": ([_P, ctypes.POINTER(PoolStatsT)], _I),
    "exaca_pool_run_plain": ([_P, _I, _I, ctypes.POINTER(_I)], _I),
    "exaca_pool_next_layer": ([_P, _I, _I], _I),
    "exaca_pool_copy_out": ([_P, _I, _P, _P], _I),
    "exaca_pool_copy_out_concurrent": ([_P, _I, _P, _P], _I),
    "exaca_pool_copy_octahedra": ([_P, _I, _P, _P, _P], _I),
    "exaca_pool_retire": ([_P, _I], _I),
    "exaca_pool_bytes_in_use": ([_P], ctypes.c_int64),
    "exaca_pool_write_outputs": ([_P, _I, _P, ctypes.c_char_p], _I),
    "exaca_problem_write_outputs": ([_P, _P, ctypes.c_char_p, _I], _I),
    "exaca_pool_last_run_ms": ([_P], ctypes.c_double),
    "exaca_pool_profile_cycles": ([_P, _I, ctypes.POINTER(ctypes.c_double)], _I),
    "exaca_pool_timed_step": ([_P, _I, ctypes.POINTER(ctypes.c_double)], _I),
    "exaca_pool_profile_persistent": ([_P, _I, ctypes.POINTER(ctypes.c_double)], _I),
    "exaca_pool_check_bounded_wait": ([_P, ctypes.POINTER(ctypes.c_int)], _I),
    "exaca_pool_run_all": ([_P, _I, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)], _I),
    "exaca_pool_status_many": ([_P, _I, ctypes.POINTER(_I), ctypes.POINTER(DomainStatus)], _I),
    "exaca_pool_grain_stats": ([_P, _I, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(GrainStatsT)], _I),
    "exaca_pool_set_config": ([_P, _I], _I),
    "exaca_pool_set_grid": ([_P, _I], _I),
    "exaca_pool_autotune": ([_P, _I, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double)], _I),
    "exaca_problem_pin": ([_P], _I),
    "exaca_census_cells": ([_I, _P, ctypes.POINTER(CellFieldsT), _I, ctypes.POINTER(CensusT)], _I),
}

_lib = None


def load_library() -> ctypes.CDLL:
    """Loads lib/libexaca_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ExacaError(-5, f"native library missing: {LIB_PATH} (run exaca_b200.build.build())")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise ExacaError(rc, load_library().exaca_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def run_program(input_file: str, device: int = 0) -> None:
    """RunProgram_Reduced at one rank (src/runCA.cpp:19-461): solve an input file, write outputs."""
    _check(load_library().exaca_run_program(os.fsencode(input_file), device))


def census_cells(device: int, domains: list, stream: int = 0) -> list:
    """exaca_census_cells: IntermediateOutputAndCheck's census (src/CAupdate.cpp:738-808) of cell
    fields already in device memory, without allocating device memory. Each domain is a dict with
    the device addresses (ints) "cell_type" (int8), "layer_id" (int8), "crit_time_step" (int32) and
    "domain_size", "active_size", "cycle", and optionally "layer" (the current layer, default 0) and
    "window_start" (first cell of the active window, default 0); at most CENSUS_MAX_DOMAINS per
    call. `stream` is a cudaStream_t handle (0: the legacy default stream); the call waits for it."""
    n = len(domains)
    arr = (CellFieldsT * max(n, 1))()
    for i, d in enumerate(domains):
        arr[i] = CellFieldsT(d["cell_type"], d["layer_id"], d["crit_time_step"], d["domain_size"],
                             d["active_size"], d["cycle"], d.get("layer", 0), d.get("window_start", 0))
    out = (CensusT * max(n, 1))()
    _check(load_library().exaca_census_cells(device, ctypes.c_void_p(stream), arr, n, out))
    return [{k: getattr(out[i], k) for k, _ in CensusT._fields_} for i in range(n)]


# Inconel625 material values (the material file shipped under data/Materials)
INCONEL625 = dict(A=-0.00000010302, B=0.00010533, C=0.0022196, D=0.0, freezing_range=210.0)


class Problem:
    """An initialised ExaCA problem (host side), from an input file or synthetic type-C parameters."""

    def __init__(self, handle):
        self._h = handle
        g = ProblemGeometry()
        _check(load_library().exaca_problem_info(self._h, ctypes.byref(g)))
        self.geometry = g

    @classmethod
    def from_file(cls, path: str) -> "Problem":
        h = ctypes.c_void_p()
        _check(load_library().exaca_problem_from_file(os.fsencode(path), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def directional(cls, nx, ny, nz, G, R, n_ratio=25, nucleation_density=10.0, dTN=5.0, dTsigma=0.5,
                    fract_surface_active=0.08, cell_size_um=1.0, material=INCONEL625) -> "Problem":
        p = DirsParams(nx=nx, ny=ny, nz=nz, cell_size_um=cell_size_um, G=G, R=R, n_ratio=n_ratio,
                       nucleation_density=nucleation_density, dTN=dTN, dTsigma=dTsigma,
                       fract_surface_active=fract_surface_active, **material)
        h = ctypes.c_void_p()
        _check(load_library().exaca_problem_directional(ctypes.byref(p), ctypes.byref(h)))
        return cls(h)

    @property
    def shape(self):
        """(nz, mx, my): the cell index is k*mx*my + i*my + j."""
        g = self.geometry
        return (g.nz, g.mx, g.my)

    def fields(self) -> dict:
        n = self.geometry.domain_size
        out = {k: np.empty(n, np.int32) for k in ("cell_type", "grain_id", "crit_time_step", "layer_id")}
        out["undercooling_change"] = np.empty(n, np.float32)
        _check(load_library().exaca_problem_fields(
            self._h, _ptr(out["cell_type"]), _ptr(out["grain_id"]), _ptr(out["crit_time_step"]),
            _ptr(out["undercooling_change"]), _ptr(out["layer_id"])))
        return out

    def slot_bytes(self) -> int:
        return int(load_library().exaca_problem_slot_bytes(self._h))

    def write_outputs(self, grain_id: np.ndarray, prefix: str, threads: int = 0) -> None:
        """The .vtk / _Misorientations.vtk files the problem's print flags ask for, from a host GrainID
        (the layout of Pool.copy_out), formatted on `threads` host threads (0: all)."""
        gid = np.ascontiguousarray(grain_id, dtype=np.int32)
        if gid.size != self.geometry.domain_size:
            raise ValueError(f"GrainID has {gid.size} cells, the problem {self.geometry.domain_size}")
        _check(load_library().exaca_problem_write_outputs(self._h, _ptr(gid), os.fsencode(prefix), int(threads)))

    def pin(self) -> None:
        """Page-locks the host fields so admission copies run at full PCIe bandwidth."""
        _check(load_library().exaca_problem_pin(self._h))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.exaca_problem_free(self._h)
            self._h = None


@dataclass
class Status:
    cycle: int
    done: bool
    nn: int
    error: int
    liquid: int
    layer: int = 0
    window_z_lo: int = 0
    window_nz: int = 0


class Pool:
    """Device pool of independent domains stepped together (one domain = the plain solver)."""

    def __init__(self, device: int = 0, budget_bytes: int = 2**62, list_capacity: int = 1 << 24):
        self._h = ctypes.c_void_p()
        _check(load_library().exaca_pool_create(device, budget_bytes, list_capacity, ctypes.byref(self._h)))
        self._problems = {}

    def admit(self, problem: Problem, device_check: bool = True) -> int:
        slot = ctypes.c_int()
        _check(load_library().exaca_pool_admit(self._h, problem._h, int(device_check), ctypes.byref(slot)))
        self._problems[slot.value] = problem
        return slot.value

    def step(self, n_cycles: int) -> None:
        _check(load_library().exaca_pool_step(self._h, n_cycles))

    def status(self, slot: int) -> Status:
        s = DomainStatus()
        _check(load_library().exaca_pool_status(self._h, slot, ctypes.byref(s)))
        return Status(s.cycle, bool(s.done), s.nn, s.error, s.liquid, s.layer, s.window_z_lo, s.window_nz)

    def grain_stats(self, slot: int, region=None) -> dict:
        """Grain statistics of the reference analysis for a slot, computed on the device; region =
        (xmin, xmax, ymin, ymax, zmin, zmax) in .vtk coordinates, None for the interior."""
        out = GrainStatsT()
        reg = None if region is None else (ctypes.c_int32 * 6)(*region)
        _check(load_library().exaca_pool_grain_stats(self._h, slot, reg, ctypes.byref(out)))
        d = {k: getattr(out, k) for k, _ in GrainStatsT._fields_ if k != "misorientation_hist"}
        d["misorientation_hist"] = list(out.misorientation_hist)
        return d

    def status_many(self, slots) -> list:
        """status() of several slots with one device read."""
        n = len(slots)
        arr = (_I * max(n, 1))(*slots)
        out = (DomainStatus * max(n, 1))()
        _check(load_library().exaca_pool_status_many(self._h, n, arr, out))
        return [Status(s.cycle, bool(s.done), s.nn, s.error, s.liquid, s.layer, s.window_z_lo, s.window_nz)
                for s in out[:n]]

    def stats(self) -> dict:
        s = PoolStatsT()
        _check(load_library().exaca_pool_stats(self._h, ctypes.byref(s)))
        return {n: getattr(s, n) for n, _ in PoolStatsT._fields_}

    def census(self, slot: int) -> dict:
        c = CensusT()
        _check(load_library().exaca_pool_census(self._h, slot, ctypes.byref(c)))
        return {n: getattr(c, n) for n, _ in CensusT._fields_}

    def run_plain(self, slot: int, verbose: bool = False) -> int:
        c = ctypes.c_int()
        _check(load_library().exaca_pool_run_plain(self._h, slot, int(verbose), ctypes.byref(c)))
        return c.value

    def next_layer(self, slot: int, verbose: bool = False) -> None:
        """DomainShiftAndResize + LayerSetup of a multilayer slot (src/runCA.cpp:344-390)."""
        _check(load_library().exaca_pool_next_layer(self._h, slot, int(verbose)))

    def copy_out(self, slot: int):
        n = self._problems[slot].geometry.domain_size
        gid = np.empty(n, np.int32)
        ct = np.empty(n, np.int32)
        _check(load_library().exaca_pool_copy_out(self._h, slot, _ptr(gid), _ptr(ct)))
        return gid, ct

    def copy_out_concurrent(self, slot: int):
        """copy_out of a slot whose domain has ended (per the last status): does not wait for cycles
        launched since, so finished results can be fetched while the next cycles run."""
        n = self._problems[slot].geometry.domain_size
        gid = np.empty(n, np.int32)
        ct = np.empty(n, np.int32)
        _check(load_library().exaca_pool_copy_out_concurrent(self._h, slot, _ptr(gid), _ptr(ct)))
        return gid, ct

    def copy_octahedra(self, slot: int):
        """Octahedron state of the current layer's active window (DL, DOCenter x3, CDL x26 per cell)."""
        s = DomainStatus()
        _check(load_library().exaca_pool_status(self._h, slot, ctypes.byref(s)))
        g = self._problems[slot].geometry
        a = g.mx * g.my * s.window_nz
        dl = np.empty(a, np.float32)
        doc = np.empty(3 * a, np.float32)
        cdl = np.empty(26 * a, np.float32)
        _check(load_library().exaca_pool_copy_octahedra(self._h, slot, _ptr(dl), _ptr(doc), _ptr(cdl)))
        return dl, doc, cdl

    def last_run_ms(self) -> float:
        """CUDA-event device time of the last run_plain on this pool."""
        return float(load_library().exaca_pool_last_run_ms(self._h))

    def profile_cycles(self, n_cycles: int) -> dict:
        """n_cycles cycles pass by pass as separate kernels; summed CUDA-event ms per pass."""
        t = (ctypes.c_double * 4)()
        _check(load_library().exaca_pool_profile_cycles(self._h, n_cycles, t))
        return {"k_step_begin": t[0], "k_grow": t[1], "k_claim": t[2], "k_capture_pass": t[3]}

    def check_bounded_wait(self) -> int:
        """The persistent kernel's grid-wide wait run where nothing can release it: returns the device
        error flags it left (FLAG_BARRIER after its 1 s limit; they are cleared again)."""
        f = ctypes.c_int()
        _check(load_library().exaca_pool_check_bounded_wait(self._h, ctypes.byref(f)))
        return int(f.value)

    def profile_persistent(self, n_cycles: int) -> dict:
        """step(n_cycles) with the persistent kernel's timeline on; per-cycle averages (us)."""
        t = (ctypes.c_double * 7)()
        _check(load_library().exaca_pool_profile_persistent(self._h, n_cycles, t))
        return {"grow_first": t[0], "grow_last": t[1], "claim_first": t[2], "claim_last": t[3], "capture_first": t[4],
                "capture_last": t[5], "cycle_end_and_start": t[6]}

    def run_all(self, chunk_cycles: int = 1000, max_cycles: int = 10**7) -> int:
        """Steps all admitted domains (device_check=True) until each has terminated; returns cycles."""
        n = ctypes.c_int64()
        _check(load_library().exaca_pool_run_all(self._h, chunk_cycles, max_cycles, ctypes.byref(n)))
        return n.value

    def set_config(self, config: int) -> None:
        _check(load_library().exaca_pool_set_config(self._h, config))

    def set_grid(self, divisor: int) -> None:
        """Persistent kernel grid: divisor d in 1-32 runs 1/d of the co-resident blocks, 0 the pool's own choice."""
        _check(load_library().exaca_pool_set_grid(self._h, divisor))

    def autotune(self, trial_cycles: int = 100):
        """Times every step configuration on trial_cycles real cycles; keeps and returns the fastest
        (config, ms per cycle of every configuration)."""
        c = ctypes.c_int()
        t = (ctypes.c_double * STEP_CONFIGS)()
        _check(load_library().exaca_pool_autotune(self._h, trial_cycles, ctypes.byref(c), t))
        return c.value, list(t)

    def timed_step(self, n_cycles: int) -> float:
        """step(n_cycles) (one persistent launch) timed with CUDA events; waits; returns ms."""
        ms = ctypes.c_double()
        _check(load_library().exaca_pool_timed_step(self._h, n_cycles, ctypes.byref(ms)))
        return ms.value

    def retire(self, slot: int) -> None:
        _check(load_library().exaca_pool_retire(self._h, slot))
        self._problems.pop(slot, None)

    def bytes_in_use(self) -> int:
        return int(load_library().exaca_pool_bytes_in_use(self._h))

    def write_outputs(self, slot: int, prefix: str) -> None:
        _check(load_library().exaca_pool_write_outputs(self._h, slot, self._problems[slot]._h, os.fsencode(prefix)))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.exaca_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
