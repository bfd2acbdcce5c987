"""Edge inputs without stored fixtures. The reference itself (its unmodified sources compiled here
against single-rank shims, oracle/_ref) runs on each; this solver's host initialisation must
reproduce its post-init fields, its output writer the reference's .vtk files from the reference's
final GrainID, and the CPU restatement oracle its final GrainID / CellType and cycle, bit for bit (no GPU; skipped where the reference was not built). On a GPU the CUDA path
must then equal the restatement on the same inputs. Cases: no substrate seeds (growth from nuclei
only), every surface site active, a domain of 3 cells a side, a flat uneven box, one small spot,
and a spot melt with dense nucleation; on the host only, spot melts of two and five layers and
type-R problems with one file repeated over layers and with a one-cell layer offset."""
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest
from helpers import INPUTS, REF_SERIAL, resolve_temperature_path, to_whole
from oracle_port import Oracle

import exaca_b200 as ex

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_golden  # noqa: E402  (debug_variant, parse_vtk)

DATA = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "exaca_b200", "data")

CASES = {
    "no_seeds": ("SmallDirS", {"Domain size in x": "24", "Domain size in y": "24", "Domain size in z": "24",
                               "Fraction of surface sites active": "0",
                               "Heterogeneous nucleation density": "3000"}),
    "all_seeds": ("SmallDirS", {"Domain size in x": "20", "Domain size in y": "20", "Domain size in z": "20",
                                "Fraction of surface sites active": "1"}),
    "three_cells": ("SmallDirS", {"Domain size in x": "3", "Domain size in y": "3", "Domain size in z": "3",
                                  "Fraction of surface sites active": "0.5",
                                  "Heterogeneous nucleation density": "100000"}),
    "flat_box": ("SmallDirS", {"Domain size in x": "40", "Domain size in y": "7", "Domain size in z": "13",
                               "Fraction of surface sites active": "0.1",
                               "Heterogeneous nucleation density": "1000"}),
    "small_spot": ("SmallSpotMelt", {"Number of spots in y": "1", "Radii of spots": "6",
                                     "Offset between spot centers": "6", "Substrate grain spacing": "4"}),
    "dense_nuclei_spot": ("SmallSpotMelt", {"Radii of spots": "10", "Offset between spot centers": "10",
                                            "Heterogeneous nucleation density": "20000"}),
}
# Several layers and temperature-file series, checked on the host only (the CUDA path's multilayer
# and type-R parity runs on the stored fixtures and on seeded random problems against the oracle)
LAYERED_CASES = {
    "spot_two_layers": ("SpotMelt3Layers", {"Number of layers": "2", "Offset between layers": "3",
                                            "Number of spots in x": "1", "Radii of spots": "7",
                                            "Offset between spot centers": "7", "Substrate grain spacing": "4"}),
    "spot_five_thin_layers": ("SpotMelt3Layers", {"Number of layers": "5", "Offset between layers": "2",
                                                  "Heterogeneous nucleation density": "2000"}),
    "r_one_file_two_layers": ("RTrackH2", {"Number of layers": "2", "Offset between layers": "3"}),
    "r_layer_offset_one": ("RTwoFiles3Layers", {"Offset between layers": "1"}),
}


def write_variant(base, changes, path):
    out = []
    for ln in open(os.path.join(INPUTS, base + ".txt")).read().splitlines():
        for key, value in changes.items():
            if ln.startswith(key):
                ln = ln[: ln.rfind(":") + 1] + " " + value
        out.append(resolve_temperature_path(ln))
    open(path, "w").write("\n".join(out) + "\n")


def run_reference(inp, work):
    """Post-init fields (the reference's debug dump), final GrainID / CellType, final cycle and the
    prefix of the output files it wrote."""
    dbg_inp = os.path.join(work, "debug_input.txt")
    make_golden.debug_variant(inp, dbg_inp, work)
    base = next(ln.split(":", 1)[1].strip() for ln in open(inp) if ln.startswith("Output file base name"))
    dump = os.path.join(work, "dump")
    os.makedirs(dump)
    env = dict(os.environ, EXACA_SHIM_DUMP_DIR=dump, EXACA_DATA_DIR=DATA)
    subprocess.run([REF_SERIAL, dbg_inp], cwd=work, env=env, capture_output=True, text=True, check=True,
                   timeout=900)
    dbg = make_golden.parse_vtk(os.path.join(work, base + "_debug.vtk"))
    cycle = int(re.search(r"output written at cycle (\d+)", open(os.path.join(work, base + ".log")).read()).group(1))
    gid = np.fromfile(os.path.join(dump, "GrainID.bin"), np.int32)
    ct = np.fromfile(os.path.join(dump, "CellType.bin"), np.int32).astype(np.int8)
    return dbg, gid, ct, cycle, os.path.join(work, base)


@pytest.mark.skipif(not os.path.exists(REF_SERIAL), reason="the reference was not built here (make -C oracle ref)")
@pytest.mark.parametrize("case", sorted(CASES) + sorted(LAYERED_CASES))
def test_edge_input_matches_reference(lib, case):
    base, changes = CASES.get(case) or LAYERED_CASES[case]
    work = tempfile.mkdtemp(prefix=f"edge_{case}_")
    try:
        inp = os.path.join(work, "input.txt")
        write_variant(base, changes, inp)
        dbg, ref_gid, ref_ct, ref_cycle, ref_prefix = run_reference(inp, work)

        # host initialisation of this solver
        p = ex.Problem.from_file(inp)
        f = p.fields()
        shape = p.shape
        assert np.array_equal(to_whole(f["cell_type"], shape), dbg["CellType"].astype(np.int8))
        assert np.array_equal(to_whole(f["crit_time_step"], shape), dbg["CritTimeStep"].astype(np.int32))
        assert np.array_equal(to_whole(f["layer_id"], shape), dbg["LayerID"].astype(np.int8))
        assert np.allclose(to_whole(f["undercooling_change"], shape), dbg["UndercoolingChange"], atol=5e-7, rtol=0)
        gid = to_whole(f["grain_id"], shape)
        pending = gid == ex.VORONOI_PENDING  # type S baseplate grains are assigned on the device
        assert np.array_equal(gid[~pending], dbg["GrainID"].astype(np.int32)[~pending])

        # output files written from the reference's final GrainID: the reference's bytes
        ours = os.path.join(work, "ours")
        p.write_outputs(ref_gid, ours)
        for suffix in (".vtk", "_Misorientations.vtk"):
            assert os.path.exists(ref_prefix + suffix)
            assert open(ours + suffix, "rb").read() == open(ref_prefix + suffix, "rb").read(), suffix

        # the CPU restatement oracle, run to the end
        o = Oracle(inp)
        assert o.run() == ref_cycle
        fo = o.fields()
        assert np.array_equal(fo["grain_id"], ref_gid)
        assert np.array_equal(fo["cell_type"].astype(np.int8), ref_ct)
    finally:
        shutil.rmtree(work, ignore_errors=True)


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_edge_input_gpu_matches_restatement(lib, tmp_path, case):
    # the restatement is pinned to the reference on these inputs by the test above
    base, changes = CASES[case]
    inp = str(tmp_path / "input.txt")
    write_variant(base, changes, inp)
    o = Oracle(inp)
    cycle = o.run()
    f = o.fields()
    p = ex.Problem.from_file(inp)
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    try:
        slot = pool.admit(p, device_check=False)
        assert pool.run_plain(slot) == cycle
        gid, ct = pool.copy_out(slot)
        dl, _, _ = pool.copy_octahedra(slot)
        assert pool.status(slot).error == 0
    finally:
        pool.close()
    assert np.array_equal(ct, f["cell_type"]), f"{np.sum(ct != f['cell_type'])} CellType differ"
    assert np.array_equal(gid, f["grain_id"]), f"{np.sum(gid != f['grain_id'])} GrainID differ"
    assert np.array_equal(dl, f["dl"]), f"{np.sum(dl != f['dl'])} DiagonalLength differ"
