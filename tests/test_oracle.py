"""The CPU restatement oracle pinned against the reference itself (golden fixtures made by the
unmodified reference sources): final GrainID, CellType, cycle, DiagonalLength / DOCenter /
CritDiagonalLength hashes, and post-init CellType. No GPU."""
import hashlib

import numpy as np
import pytest

from helpers import golden_cases, input_path, load_golden, to_whole
from oracle_port import Oracle


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# the serial restatement on the small cases (the large ones take it many minutes)
@pytest.mark.parametrize("case", golden_cases(dense_only=True))
def test_oracle_matches_reference(case):
    g = load_golden(case)
    o = Oracle(input_path(case))
    f0 = o.fields()
    shape = (o.nz, o.mx, o.my)
    assert np.array_equal(to_whole(f0["cell_type"], shape), g["init_cell_type"])
    assert np.array_equal(to_whole(f0["grain_id"], shape), g["init_grain_id"])
    cycle = o.run()
    assert cycle == int(g["cycle"])
    f = o.fields()
    assert np.array_equal(f["grain_id"], g["final_grain_id"])
    assert np.array_equal(f["cell_type"].astype(np.int8), g["final_cell_type"])
    assert sha(f["dl"]) == str(g["sha_dl"])
    ever = f["dl"] != 0
    assert sha(f["doc"].reshape(-1, 3)[ever]) == str(g["sha_doc"])
    assert sha(f["cdl"].reshape(-1, 26)[ever]) == str(g["sha_cdl"])
