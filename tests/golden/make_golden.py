"""Generate the golden fixtures of the parity tests from the ExaCA reference itself.

Runs the UNMODIFIED reference sources, compiled against the single-rank shims by
`make -C oracle ref` (Serial dispatch = the reference's deterministic loop order), on every input in
tests/golden/inputs/, and stores per case in tests/golden/<case>.npz:

  init_*       cell fields after initialisation, from the reference's own debug dump (_debug.vtk,
               PrintDebug = 2): CellType, GrainID, CritTimeStep, LayerID, Melted, UndercoolingChange
               on the whole-domain grid (nz, ny, nx) the reference prints
  final_*      GrainID and CellType (full rank-local arrays) at the end of the run,
               captured by the shim when the reference releases its views
  sha_*        SHA-256 of the reference's .vtk and _Misorientations.vtk output files, of the final
               DiagonalLength array (for multilayer runs: of the last layer's active window), and of
               DOCenter / CritDiagonalLength over cells with DL != 0
  cycle        the final cycle written to the .log
  census       the reference's every-1000-cycle stdout lines
  log          the reference's .log file (its timing values vary from run to run)
  stdout       the reference's whole stdout

Cases of more than DENSE_LIMIT cells store digests of the dense arrays instead (digest_only).

Needs the reference sources (build container only; oracle/Makefile REF). Usage:
    python tests/golden/make_golden.py [case ...]
"""
import hashlib
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
INPUTS = os.path.join(HERE, "inputs")
REF = os.path.join(ROOT, "oracle", "_ref", "ExaCA-ref-serial")


def debug_variant(src, dst, outdir):
    lines = open(src).read().splitlines()
    out = []
    for ln in lines:
        if ln.startswith("Path to output"):
            ln = "Path to output: " + outdir + "/"
        if "Print data for main Kokkos views" in ln or "Print data for all main data structures" in ln:
            ln = ln[: ln.rfind(":") + 1] + " Y"
        if ln.startswith("Path to temperature file"):
            # relative to tests/golden/inputs (the reference resolves it against its working directory)
            key, rel = ln.split(":", 1)
            ln = key + ": " + os.path.join(INPUTS, rel.strip())
        out.append(ln)
    open(dst, "w").write("\n".join(out) + "\n")


def parse_vtk(path):
    """Returns {name: array (nz, ny, nx)} of a legacy ASCII STRUCTURED_POINTS file."""
    with open(path) as f:
        text = f.read()
    dims = tuple(int(v) for v in re.search(r"DIMENSIONS (\d+) (\d+) (\d+)", text).groups())
    nx, ny, nz = dims
    blocks = {}
    parts = re.split(r"SCALARS (\S+) (int|float) 1\nLOOKUP_TABLE default\n", text)
    for q in range(1, len(parts), 3):
        name, typ, body = parts[q], parts[q + 1], parts[q + 2]
        vals = np.array(body.split(), dtype=np.float64 if typ == "float" else np.int64)
        key = name
        while key in blocks:
            key += "_2"
        blocks[key] = vals.reshape(nz, ny, nx)
    return blocks


def sha(b):
    return hashlib.sha256(b).hexdigest()


# Cases above this many cells keep SHA-256 digests of their dense fields instead of the fields
# (key "sha_<field>", of the array in the dtype listed here), so the fixtures stay small;
# UndercoolingChange keeps the digest of where it is non-zero and its distinct non-zero values.
DENSE_LIMIT = 2_000_000
DENSE_DTYPES = dict(init_cell_type=np.int8, init_grain_id=np.int32, init_cts=np.int32, init_layer_id=np.int8,
                    init_melted=np.int8, final_grain_id=np.int32, final_cell_type=np.int8)


def digest_only(out):
    small = {k: v for k, v in out.items() if k not in DENSE_DTYPES and k != "init_du"}
    for k, dt in DENSE_DTYPES.items():
        small["sha_" + k] = sha(np.ascontiguousarray(out[k], dtype=dt).tobytes())
        small["shape_" + k] = np.array(out[k].shape, np.int64)
    du = out["init_du"]
    small["sha_init_du_nonzero"] = sha(np.ascontiguousarray(du != 0).tobytes())
    small["init_du_values"] = np.unique(du[du != 0]).astype(np.float32)
    return small


def run_case(case):
    src = os.path.join(INPUTS, case + ".txt")
    base = None
    for ln in open(src):
        if ln.startswith("Output file base name"):
            base = ln.split(":", 1)[1].strip()
    work = tempfile.mkdtemp(prefix="golden_")
    try:
        inp = os.path.join(work, "input.txt")
        debug_variant(src, inp, work)
        dump = os.path.join(work, "dump")
        os.makedirs(dump)
        env = dict(os.environ, EXACA_SHIM_DUMP_DIR=dump)
        r = subprocess.run([REF, inp], cwd=work, env=env, capture_output=True, text=True, check=True)
        dbg = parse_vtk(os.path.join(work, base + "_debug.vtk"))
        # census and jump lines, in order (a census line may follow text printed without a line break)
        census = [m.group(0) for m in re.finditer(r"cycle = \d+ Superheated.*|^Jumping to cycle \d+", r.stdout,
                                                  re.MULTILINE)]
        log = open(os.path.join(work, base + ".log")).read()
        cycle = int(re.search(r"output written at cycle (\d+)", log).group(1))
        gid = np.fromfile(os.path.join(dump, "GrainID.bin"), np.int32)
        ct = np.fromfile(os.path.join(dump, "CellType.bin"), np.int32)
        # multilayer: the octahedron views were resized, and their final storage is the dump before
        # the host mirror's (which still holds the first layer's window)
        layers = 1
        for ln in open(src):
            if ln.startswith("Number of layers"):
                layers = int(ln.split(":", 1)[1])
        octa = ".prev.bin" if layers > 1 else ".bin"
        dl = np.fromfile(os.path.join(dump, "DiagonalLength" + octa), np.float32)
        doc = np.fromfile(os.path.join(dump, "DOCenter" + octa), np.float32).reshape(-1, 3)
        cdl = np.fromfile(os.path.join(dump, "CritDiagonalLength" + octa), np.float32).reshape(-1, 26)
        ever = dl != 0
        out = dict(
            init_cell_type=dbg["CellType"].astype(np.int8),
            init_grain_id=dbg["GrainID"].astype(np.int32),
            init_cts=dbg["CritTimeStep"].astype(np.int32),
            init_layer_id=dbg["LayerID"].astype(np.int8),
            init_melted=dbg["Melted"].astype(np.int8),
            init_du=dbg["UndercoolingChange"].astype(np.float32),
            final_grain_id=gid,
            final_cell_type=ct.astype(np.int8),
            sha_vtk=sha(open(os.path.join(work, base + ".vtk"), "rb").read()),
            sha_mis=sha(open(os.path.join(work, base + "_Misorientations.vtk"), "rb").read()),
            sha_dl=sha(dl.tobytes()),
            sha_doc=sha(np.ascontiguousarray(doc[ever]).tobytes()),
            sha_cdl=sha(np.ascontiguousarray(cdl[ever]).tobytes()),
            cycle=np.int64(cycle),
            census=np.array(census),
            log=np.array(log),
            stdout=np.array(r.stdout),
        )
        if gid.size > DENSE_LIMIT:
            out = digest_only(out)
        np.savez_compressed(os.path.join(HERE, case + ".npz"), **out)
        print(f"{case}: cycle {cycle}, {gid.size} cells, {len(census)} census lines")
    finally:
        shutil.rmtree(work, ignore_errors=True)


def main():
    if not os.path.exists(REF):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "-j8"], check=True)
    cases = sys.argv[1:] or sorted(f[:-4] for f in os.listdir(INPUTS) if f.endswith(".txt"))
    for c in cases:
        run_case(c)


if __name__ == "__main__":
    main()
