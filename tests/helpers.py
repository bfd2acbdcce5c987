"""Shared helpers of the parity tests (test infrastructure)."""
import hashlib
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
INPUTS = os.path.join(GOLDEN, "inputs")
REF_SERIAL = os.path.join(ROOT, "oracle", "_ref", "ExaCA-ref-serial")


def reference_error(path):
    """The exception message of the reference (compiled against single-rank shims in oracle/_ref)
    on this input file, run from the file's folder: '' when it initialises and runs to the end, None
    when the reference was not built here."""
    if not os.path.exists(REF_SERIAL):
        return None
    r = subprocess.run([REF_SERIAL, os.path.basename(path)], cwd=os.path.dirname(path), capture_output=True,
                       text=True, timeout=600,
                       env=dict(os.environ, EXACA_DATA_DIR=os.path.join(ROOT, "exaca_b200", "data")))
    for ln in (r.stdout + r.stderr).splitlines():
        if "what():" in ln:
            return ln.split("what():", 1)[1].strip()
    assert r.returncode == 0, r.stderr[-2000:]
    return ""


def golden_cases(dense_only=False):
    """Golden fixture names; dense_only: the cases that store their dense fields (small domains),
    for tests that need the arrays themselves or run the serial restatement on them."""
    cases = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    return [c for c in cases if is_dense(load_golden(c))] if dense_only else cases


# dtype of each dense golden field, in which its digest is taken for the large cases (make_golden.py)
DENSE_DTYPES = dict(init_cell_type=np.int8, init_grain_id=np.int32, init_cts=np.int32, init_layer_id=np.int8,
                    init_melted=np.int8, final_grain_id=np.int32, final_cell_type=np.int8)


def is_dense(g):
    return "final_grain_id" in g.files


def field_equal(g, name, arr):
    """arr equals the golden field `name`: the stored array, or for large cases its shape and the
    SHA-256 digest of its bytes in the field's dtype."""
    if name in g.files:
        return np.array_equal(arr, g[name])
    a = np.ascontiguousarray(arr, dtype=DENSE_DTYPES[name])
    return tuple(a.shape) == tuple(g["shape_" + name]) and hashlib.sha256(a.tobytes()).hexdigest() == str(g["sha_" + name])


def load_golden(case):
    return np.load(os.path.join(GOLDEN, case + ".npz"))


def resolve_temperature_path(line):
    """Temperature-file paths of the golden inputs are relative to tests/golden/inputs; the solver
    (like the reference) resolves them against the working directory, so copies get absolute ones."""
    if line.startswith("Path to temperature file"):
        key, rel = line.split(":", 1)
        return key + ": " + os.path.join(INPUTS, rel.strip())
    return line


def input_path(case):
    src = os.path.join(INPUTS, case + ".txt")
    lines = open(src).read().splitlines()
    if not any(ln.startswith("Path to temperature file") for ln in lines):
        return src
    dst = os.path.join(tempfile.gettempdir(), f"exaca_golden_{os.getpid()}_{case}.txt")
    open(dst, "w").write("\n".join(resolve_temperature_path(ln) for ln in lines) + "\n")
    return dst


def to_whole(a, shape):
    """Rank-local array (nz, mx, my) -> the reference's whole-domain print grid (nz, ny, nx),
    ghost ring dropped, planes k = 0 and nz - 1 zeroed (src/CAprint.cpp:18-29, 285-346)."""
    nz, mx, my = shape
    w = a.reshape(nz, mx, my)[:, 1:-1, 1:-1].transpose(0, 2, 1).copy()
    w[0] = 0
    w[-1] = 0
    return w


def copy_input(case, outdir):
    """Copy of an input file whose outputs go to outdir."""
    lines = open(input_path(case)).read().splitlines()
    out = []
    for ln in lines:
        if ln.startswith("Path to output"):
            ln = "Path to output: " + outdir + "/"
        out.append(resolve_temperature_path(ln))
    dst = os.path.join(outdir, case + ".txt")
    open(dst, "w").write("\n".join(out) + "\n")
    return dst


def output_base(case):
    for ln in open(input_path(case)):
        if ln.startswith("Output file base name"):
            return ln.split(":", 1)[1].strip()
    raise KeyError(case)
