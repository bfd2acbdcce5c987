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
    """Caller-owned device copies of a slot's CellType (read back from the device) and of its LayerID
    and CritTimeStep. The reference assigns LayerID and CritTimeStep to every cell of every layer at
    initialisation and never changes them (the layer loop, src/runCA.cpp:344-405, moves the window
    only), so the problem's initial fields are the slot's; CellType changes every cycle."""
    _, ct = pool.copy_out(slot)
    f = prob.fields()
    t = {
        "cell_type": torch.from_numpy(ct.astype(np.int8)).cuda(),
        "layer_id": torch.from_numpy(f["layer_id"].astype(np.int8)).cuda(),
        "crit_time_step": torch.from_numpy(f["crit_time_step"]).cuda(),
    }
    keep.append(t)  # the tensors outlive the census call
    g = prob.geometry
    st = pool.status(slot)
    plane = g.mx * g.my
    d = {k: v.data_ptr() for k, v in t.items()}
    d.update(domain_size=g.domain_size, active_size=st.window_nz * plane, cycle=st.cycle, layer=st.layer,
             window_start=st.window_z_lo * plane)
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


@pytest.mark.gpu
def test_census_cells_in_a_later_layer(lib):
    """A three-layer spot melt stepped into its second layer: the layer number selects the cells that
    are classified (the first layer's are neither counted nor remaining once solid), and the window
    start bounds the cells the next CritTimeStep is taken over; both must equal the pool's census."""
    import torch

    prob = ex.Problem.from_file(input_path("SpotMelt3Layers"))
    pool = ex.Pool(0, list_capacity=prob.geometry.domain_size)
    slot = pool.admit(prob, device_check=False)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        # layer 0 to its end as the plain driver's census finds it (idle cycles instead of its jump)
        for _ in range(200):
            pool.step(1000)
            c = pool.census(slot)
            if c["superheated"] + c["undercooled"] == 0:
                break
        else:
            pytest.fail("layer 0 did not end within 200000 cycles")
        pool.next_layer(slot)
        st = pool.status(slot)
        assert st.layer == 1 and st.window_z_lo > 0
        checked = 0
        for _ in range(60):
            pool.step(500)
            want = pool.census(slot)
            keep = []
            dom = device_domain(torch, pool, slot, prob, keep)
            assert ex.census_cells(0, [dom], stream=stream) == [want]
            assert ex.census_cells(0, [dom], stream=stream) == [want]
            if want["undercooled"] > 0 and want["active"] > 0 and want["solid"] > 0:
                checked += 1
                # the window and layer matter here: the census of layer 0 over the whole domain differs
                first = dict(dom, layer=0, window_start=0)
                assert ex.census_cells(0, [first], stream=stream) != [want]
            if checked >= 2:
                break
        assert checked >= 2, "layer 1 never held undercooled, active and solid cells together"
    finally:
        pool.close()
