"""Grain statistics of the reference's OpenMP build (nondeterministic capture order) on golden
inputs, the fixture of the 2 % statistical agreement tests. Runs oracle/_ref/ExaCA-ref-omp (the
unmodified reference compiled against the shims by `make -C oracle ref`) several times per case and
stores the statistics of every run (oracle/grain_stats.py) in tests/golden/omp_stats.json.

Needs the oracle build (build container). Usage: python tests/golden/make_omp_stats.py
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import grain_stats  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "ExaCA-ref-omp")
CASES = ["DirS64", "SmallDirS"]
RUNS = 3
THREADS = 8


def run(case):
    src = os.path.join(HERE, "inputs", case + ".txt")
    g = np.load(os.path.join(HERE, case + ".npz"))
    nz, ny, nx = g["init_melted"].shape
    melted = np.zeros((nz, nx + 2, ny + 2), np.int8)
    melted[:, 1:nx + 1, 1:ny + 1] = g["init_melted"].transpose(0, 2, 1)
    guv = np.loadtxt(os.path.join(ROOT, "exaca_b200", "data", "Substrate", "GrainOrientationVectors_Uniform10k.csv"),
                     skiprows=1, delimiter=",", dtype=np.float32)
    deltax = None
    for ln in open(src):
        if ln.startswith("Cell size"):
            deltax = float(ln.split(":", 1)[1]) * 1e-6
    out = []
    for r in range(RUNS):
        work = tempfile.mkdtemp(prefix="ompstats_")
        try:
            lines = [("Path to output: " + work + "/") if ln.startswith("Path to output") else ln
                     for ln in open(src).read().splitlines()]
            inp = os.path.join(work, "input.txt")
            open(inp, "w").write("\n".join(lines) + "\n")
            dump = os.path.join(work, "dump")
            os.makedirs(dump)
            env = dict(os.environ, EXACA_SHIM_DUMP_DIR=dump, OMP_NUM_THREADS=str(THREADS),
                       EXACA_DATA_DIR=os.path.join(ROOT, "exaca_b200", "data"))
            subprocess.run([REF, inp], cwd=work, env=env, capture_output=True, text=True, check=True)
            gid = np.fromfile(os.path.join(dump, "GrainID.bin"), np.int32)
            st = grain_stats.grain_stats(gid, melted.ravel(), guv, nx, ny, nz, deltax)
            st["identical_to_serial"] = bool(np.array_equal(gid, g["final_grain_id"]))
            out.append(st)
        finally:
            shutil.rmtree(work, ignore_errors=True)
    serial = grain_stats.grain_stats(g["final_grain_id"], melted.ravel(), guv, nx, ny, nz, deltax)
    return dict(threads=THREADS, runs=out, serial=serial)


def main():
    res = {c: run(c) for c in CASES}
    json.dump(res, open(os.path.join(HERE, "omp_stats.json"), "w"), indent=1)
    for c, v in res.items():
        print(c, [(r["n_grains"], round(r["mean_misorientation_deg"], 3), r["identical_to_serial"]) for r in v["runs"]],
              "serial", v["serial"]["n_grains"], round(v["serial"]["mean_misorientation_deg"], 3))


if __name__ == "__main__":
    main()
