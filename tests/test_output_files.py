"""Output files without a device: the .vtk and _Misorientations.vtk text written from the
reference's own final GrainID (golden fixtures) equals, byte for byte, what the reference wrote
(src/CAprint.cpp:285-460), whatever the number of host threads that format the z planes."""
import hashlib
import os

import numpy as np
import pytest

from helpers import golden_cases, input_path, load_golden, output_base

import exaca_b200 as ex


def sha_file(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


@pytest.mark.parametrize("case", golden_cases(dense_only=True))
@pytest.mark.parametrize("threads", [1, 3, 0])
def test_output_files_match_reference(case, threads, tmp_path):
    g = load_golden(case)
    p = ex.Problem.from_file(input_path(case))
    prefix = os.path.join(str(tmp_path), output_base(case))
    p.write_outputs(np.asarray(g["final_grain_id"]), prefix, threads=threads)
    assert sha_file(prefix + ".vtk") == str(g["sha_vtk"])
    assert sha_file(prefix + "_Misorientations.vtk") == str(g["sha_mis"])


def test_output_rejects_wrong_size(tmp_path):
    p = ex.Problem.from_file(input_path(golden_cases()[0]))
    with pytest.raises(ValueError):
        p.write_outputs(np.zeros(5, np.int32), os.path.join(str(tmp_path), "x"))
