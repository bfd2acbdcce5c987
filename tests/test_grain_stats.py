"""Grain statistics (the reference analysis' grain count, mean grain volume, nucleated fraction and
misorientation histogram) computed on the device, against the numpy restatement on the same field,
and within 2 % of the reference's nondeterministic OpenMP build (fixture: tests/golden/omp_stats.json
from tests/golden/make_omp_stats.py)."""
import json
import os
import sys

import numpy as np
import pytest

from helpers import input_path, load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import grain_stats as gs  # noqa: E402

import exaca_b200 as ex  # noqa: E402

OMP = json.load(open(os.path.join(ROOT, "tests", "golden", "omp_stats.json")))
GUV = np.loadtxt(os.path.join(ROOT, "exaca_b200", "data", "Substrate", "GrainOrientationVectors_Uniform10k.csv"),
                 skiprows=1, delimiter=",", dtype=np.float32)


def melted_local(g):
    nz, ny, nx = g["init_melted"].shape
    m = np.zeros((nz, nx + 2, ny + 2), np.int8)
    m[:, 1:nx + 1, 1:ny + 1] = g["init_melted"].transpose(0, 2, 1)
    return m.ravel(), nx, ny, nz


@pytest.mark.parametrize("case", sorted(OMP))
def test_reference_backends_agree_within_2_percent(case):
    # the Serial run (golden) and every OpenMP run of the reference itself
    for run in OMP[case]["runs"]:
        d = gs.agree(run, OMP[case]["serial"])
        assert d["ok"], d


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(OMP))
def test_device_grain_stats(lib, case):
    g = load_golden(case)
    p = ex.Problem.from_file(input_path(case))
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    slot = pool.admit(p, device_check=False)
    pool.run_plain(slot)
    dev = pool.grain_stats(slot)
    gid, _ = pool.copy_out(slot)
    pool.close()
    mel, nx, ny, nz = melted_local(g)
    host = gs.grain_stats(gid, mel, GUV, nx, ny, nz, 1e-6)
    for k in ("region_cells", "melted_cells", "n_grains", "misorientation_hist"):
        assert dev[k] == host[k], k
    for k in ("mean_grain_volume_um3", "nucleated_fraction", "mean_misorientation_deg", "mean_misorientation_top_deg"):
        assert dev[k] == pytest.approx(host[k], rel=1e-9), k
    # the device statistics of this (Serial-identical) run and every OpenMP run of the reference
    for run in OMP[case]["runs"]:
        d = gs.agree(dev, run)
        assert d["ok"], d
