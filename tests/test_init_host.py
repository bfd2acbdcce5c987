"""Host-side initialisation vs the reference's own post-init debug dump (no GPU needed)."""
import numpy as np
import pytest

from helpers import golden_cases, input_path, load_golden, to_whole

import exaca_b200 as ex


@pytest.mark.parametrize("case", golden_cases())
def test_init_fields_match_reference(lib, case):
    g = load_golden(case)
    p = ex.Problem.from_file(input_path(case))
    f = p.fields()
    shape = p.shape
    assert np.array_equal(to_whole(f["cell_type"], shape), g["init_cell_type"])
    assert np.array_equal(to_whole(f["crit_time_step"], shape), g["init_cts"])
    assert np.array_equal(to_whole(f["layer_id"], shape), g["init_layer_id"])
    # the debug dump prints UndercoolingChange with %f
    assert np.allclose(to_whole(f["undercooling_change"], shape), g["init_du"], atol=5e-7, rtol=0)
    gid = to_whole(f["grain_id"], shape)
    pending = gid == ex.VORONOI_PENDING
    assert np.array_equal(gid[~pending], g["init_grain_id"][~pending])
