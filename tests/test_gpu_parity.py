"""GPU solver vs the ExaCA reference (Kokkos-Serial order): bit-exact GrainID, CellType, final
cycle, octahedron state and output files, on the golden cases."""
import hashlib
import os

import numpy as np
import pytest

from helpers import copy_input, field_equal, golden_cases, input_path, load_golden, output_base, to_whole

import exaca_b200 as ex

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(b).hexdigest()


@pytest.mark.parametrize("case", golden_cases())
def test_plain_run_bit_exact(lib, case):
    g = load_golden(case)
    p = ex.Problem.from_file(input_path(case))
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    slot = pool.admit(p, device_check=False)
    # state after admission = the reference's state after initialisation
    gid0, ct0 = pool.copy_out(slot)
    assert field_equal(g, "init_grain_id", to_whole(gid0, p.shape))
    assert field_equal(g, "init_cell_type", to_whole(ct0, p.shape))
    cycle = pool.run_plain(slot)
    assert cycle == int(g["cycle"])
    gid, ct = pool.copy_out(slot)
    assert field_equal(g, "final_grain_id", gid), "GrainID differs"
    assert field_equal(g, "final_cell_type", ct.astype(np.int8)), "CellType differs"
    dl, doc, cdl = pool.copy_octahedra(slot)
    assert sha(dl.tobytes()) == str(g["sha_dl"])
    ever = dl != 0
    assert sha(np.ascontiguousarray(doc.reshape(-1, 3)[ever]).tobytes()) == str(g["sha_doc"])
    assert sha(np.ascontiguousarray(cdl.reshape(-1, 26)[ever]).tobytes()) == str(g["sha_cdl"])
    st = pool.status(slot)
    assert st.error == 0
    pool.close()


@pytest.mark.parametrize("case", golden_cases())
def test_run_program_outputs_identical(lib, case, tmp_path):
    g = load_golden(case)
    inp = copy_input(case, str(tmp_path))
    ex.run_program(inp, 0)
    base = os.path.join(str(tmp_path), output_base(case))
    assert sha(open(base + ".vtk", "rb").read()) == str(g["sha_vtk"])
    assert sha(open(base + "_Misorientations.vtk", "rb").read()) == str(g["sha_mis"])
    log = open(base + ".log").read()
    assert f"output written at cycle {int(g['cycle'])}" in log
