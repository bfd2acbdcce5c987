"""Failure detection without a GPU fault: the persistent kernel's grid-wide wait, run where nothing
can release it (one of two blocks leaves without arriving), ends by its 1 s limit with the barrier
flag set instead of hanging; the host reads the flag, and the same pool then solves a golden case
bit for bit (the context stays usable). Admission beyond the pool's HBM budget is refused before
anything is allocated."""
import time

import numpy as np
import pytest

from helpers import input_path, load_golden

import exaca_b200 as ex

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_pool_carries_on(lib):
    case = "SmallDirS"
    p = ex.Problem.from_file(input_path(case))
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    try:
        t0 = time.perf_counter()
        flags = pool.check_bounded_wait()
        waited = time.perf_counter() - t0
        assert flags == ex.FLAG_BARRIER
        assert 0.9 < waited < 60.0
        slot = pool.admit(p, device_check=False)
        cycle = pool.run_plain(slot)
        gid, ct = pool.copy_out(slot)
        assert pool.status(slot).error == 0
    finally:
        pool.close()
    g = load_golden(case)
    assert cycle == int(g["cycle"])
    assert np.array_equal(gid, g["final_grain_id"])
    assert np.array_equal(ct.astype(np.int8), g["final_cell_type"])


def test_admission_beyond_the_budget_is_refused(lib):
    p = ex.Problem.from_file(input_path("SmallDirS"))
    pool = ex.Pool(0, budget_bytes=p.slot_bytes() - 1, list_capacity=p.geometry.active_size)
    try:
        with pytest.raises(ex.ExacaError) as e:
            pool.admit(p, device_check=False)
        assert e.value.code == -4 and "HBM budget" in str(e.value)
        assert pool.bytes_in_use() == 0
    finally:
        pool.close()
