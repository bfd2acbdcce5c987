"""The grain-statistics checker (oracle/grain_stats.py) pinned against the reference's own analysis
program (analysis/src, compiled here against the single-rank shims as oracle/_ref/grain_analysis)
on the reference's own output files: grain count, mean grain volume, nucleated volume fraction,
mean misorientation to +Z over the region and its top plane, and the misorientation histogram
(from the per-cell misorientation file the analysis writes). No GPU; skipped where the reference
was not built. Type-C runs only: for types S and R the analysis looks for the number of layers at
the start of a log line (analysis/src/GAutils.cpp:110-115), while the reference's log writes "This
pattern was repeated for N layers" (src/CAprint.cpp:513), so the analysis stops on its own stoi."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from helpers import REF_SERIAL, ROOT, copy_input, output_base

sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import grain_stats as gs  # noqa: E402
import make_golden  # noqa: E402  (parse_vtk)

ANALYSIS = os.path.join(ROOT, "oracle", "_ref", "grain_analysis")
DATA = os.path.join(ROOT, "exaca_b200", "data")
ORIENTATIONS = "GrainOrientationVectors_Uniform10k.csv"
GUV = np.loadtxt(os.path.join(DATA, "Substrate", ORIENTATIONS), skiprows=1, delimiter=",", dtype=np.float32)


def analysis_file(path, base, region):
    xmin, xmax, ymin, ymax, zmin, zmax = region
    lines = [
        "Grain statistics of one run",
        "*****",
        f"Path to/name of log (.log) file associated with the microstructure of interest: {base}.log",
        f"Path to/name of microstructure (.vtk) file: {base}.vtk",
        f"Path to file of grain orientations (rotation matrix form): {ORIENTATIONS}",
        f"Path to/base (without file extension) name of data files of output resulting from this analysis: {base}",
        "**********",
        "SECTION 1: RVEs", "*****", "**********",
        "SECTION 2: cross-sections", "*****", "**********",
        "SECTION 3: representative region", "*****",
        f"X Bounds (in cells): [{xmin}, {xmax}]",
        f"Y Bounds (in cells): [{ymin}, {ymax}]",
        f"Z Bounds (in cells): [{zmin}, {zmax}]",
        "Print misorientation data (Y or N): Y",
        "Print grain volume distribution (Y or N): N",
        "Print mean aspect ratio distribution (Y or N): N",
        "Print mean grain area as a function of build height (Y or N): N",
        "Print mean weighted grain area as a function of build height (Y or N): N",
        "Print mean grain height distribution (Y or N): N",
        "Print grain width distribution at a specific build height near the top surface (Y or N): N",
        "Print volume for pole figure analysis in MTEX: N",
    ]
    open(path, "w").write("\n".join(lines) + "\n")


def number(pattern, text):
    return float(re.search(pattern, text).group(1))


@pytest.mark.skipif(not (os.path.exists(REF_SERIAL) and os.path.exists(ANALYSIS)),
                    reason="the reference and its analysis program were not built here (make -C oracle ref)")
@pytest.mark.parametrize("case", ["DirSNuc", "SmallDirS"])
def test_checker_matches_reference_analysis(tmp_path, case):
    work = str(tmp_path)
    env = dict(os.environ, EXACA_DATA_DIR=DATA)
    inp = copy_input(case, work)
    subprocess.run([REF_SERIAL, inp], cwd=work, env=env, capture_output=True, text=True, check=True, timeout=900)
    base = output_base(case)
    vtk = make_golden.parse_vtk(os.path.join(work, base + ".vtk"))
    nz, ny, nx = vtk["GrainID"].shape
    region = (1, nx - 2, 1, ny - 2, 1, nz - 2)  # the checker's default: the interior without the walls
    analysis_file(os.path.join(work, "analysis.txt"), base, region)
    r = subprocess.run([ANALYSIS, "analysis.txt"], cwd=work, env=env, capture_output=True, text=True, check=True,
                       timeout=900)
    out = r.stdout

    # the checker on the same fields, as rank-local arrays (index k * mx * my + i * my + j)
    def local(whole):
        a = np.zeros((nz, nx + 2, ny + 2), np.int64)
        a[:, 1:nx + 1, 1:ny + 1] = whole.transpose(0, 2, 1)
        return a.ravel()

    deltax = number(r"Cell size is (\S+) microns", out)
    st = gs.grain_stats(local(vtk["GrainID"]), local(vtk["Melted"]), GUV, nx, ny, nz, deltax, region)

    assert st["n_grains"] == int(number(r"There are (\d+) grains", out))
    assert st["mean_grain_volume_um3"] == pytest.approx(number(r"mean grain volume is (\S+) cubic", out), rel=1e-5)
    assert st["nucleated_fraction"] == pytest.approx(number(r"nucleated grains is (\S+)", out), rel=1e-5, abs=1e-7)
    assert st["melted_cells"] == int(number(r"cells, (\d+) underwent melting", out))
    assert st["mean_misorientation_deg"] == pytest.approx(
        number(r"\+Z direction is (\S+) degrees", out), rel=1e-5)
    top = re.search(r"region top \(Z = \d+\) is (\S+) degrees", out).group(1)
    if top not in ("nan", "-nan"):
        assert st["mean_misorientation_top_deg"] == pytest.approx(float(top), rel=1e-5)
    # histogram of the per-cell misorientations the analysis wrote (one value per melted cell)
    per_cell = np.loadtxt(os.path.join(work, base + "_MisorientationFrequency.csv"), dtype=np.float64, ndmin=1)
    hist = np.bincount(np.minimum(per_cell.astype(np.int64), gs.HIST_BINS - 1), minlength=gs.HIST_BINS)
    assert hist.tolist() == st["misorientation_hist"]
