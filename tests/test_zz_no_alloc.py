"""exaca_census_cells, the census that allocates no device memory (its working data sits in a fixed
array in the library's device image), against exaca_pool_census on the same domain state.

The cell fields are copied out of pool slots into caller-owned device tensors; the census of
those tensors must equal the pool's census of the slots, on two calls in a row (the second call
sees what the first left in the shared scratch array)."""
import numpy as np
import pytest

from helpers import input_path

import exaca_b200 as ex


def test_rejects_more_domains_than_the_scratch_holds(lib):
    with pytest.raises(ex.ExacaError) as e:
        ex.census_cells(0, [dict(cell_type=0, layer_id=0, crit_time_step=0, domain_size=0, active_size=0, cycle=0)]
                        * (ex.CENSUS_MAX_DOMAINS + 1))
    assert e.value.code == -5 and "at most" in str(e.value)
    assert ex.census_cells(0, []) == []


def device_domain(torch, pool, slot, prob, keep):
    _, ct = pool.copy_out(slot)
    f = prob.fields()
    t = {
        "cell_type": torch.from_numpy(ct.astype(np.int8)).cuda(),
        "layer_id": torch.from_numpy(f["layer_id"].astype(np.int8)).cuda(),
        "crit_time_step": torch.from_numpy(f["crit_time_step"]).cuda(),
    }
    keep.append(t)  # the tensors outlive the census call
    g = prob.geometry
    d = {k: v.data_ptr() for k, v in t.items()}
    d.update(domain_size=g.domain_size, active_size=g.active_size, cycle=pool.status(slot).cycle)
    return d


@pytest.mark.gpu
def test_census_cells_equals_pool_census_twice(lib):
    import torch

    probs = [ex.Problem.from_file(input_path("SmallDirS")),
             ex.Problem.directional(48, 40, 56, G=5e5, R=3e5, n_ratio=25, nucleation_density=200, dTN=2.0,
                                    dTsigma=0.5, fract_surface_active=0.05)]
    cap = sum(p.geometry.active_size for p in probs)
    pool = ex.Pool(0, list_capacity=cap)
    slots = [pool.admit(p, device_check=False) for p in probs]
    stream = torch.cuda.current_stream().cuda_stream
    try:
        for cycles, order in ((1500, [0, 1]), (800, [1, 0])):
            pool.step(cycles)
            keep = []
            doms = [device_domain(torch, pool, slots[i], probs[i], keep) for i in order]
            want = [pool.census(slots[i]) for i in order]
            got = ex.census_cells(0, doms, stream=stream)
            assert got == want
            # liquid, active and solid cells all present: the comparison covers every counter
            assert all(w["undercooled"] + w["superheated"] > 0 and w["active"] > 0 and w["solid"] > 0 for w in want)
            # the same call again on the state the previous call left in the scratch array
            assert ex.census_cells(0, doms, stream=stream) == want
            assert ex.census_cells(0, doms[1:], stream=0) == want[1:]
    finally:
        pool.close()
