"""GPU solver vs the CPU restatement oracle on seeded random problems of both kinds: identical
CellType, GrainID and DiagonalLength after the same raw cycle counts, and identical final state and
cycle at termination (bit-exact; the arithmetic is integer and reference-order floating point),
single-layer and multilayer (the active window moved between layers), and with temperatures read
from seeded random temperature files (type R: interpolation, file series, several cooling rates)."""
import numpy as np
import pytest

from gen_inputs import random_c, random_r, random_s
from oracle_port import Oracle

import exaca_b200 as ex

pytestmark = pytest.mark.gpu


def compare(pool, slot, o, where):
    gid, ct = pool.copy_out(slot)
    f = o.fields()
    assert np.array_equal(ct, f["cell_type"]), f"{where}: {np.sum(ct != f['cell_type'])} CellType differ"
    assert np.array_equal(gid, f["grain_id"]), f"{where}: {np.sum(gid != f['grain_id'])} GrainID differ"
    dl, doc, cdl = pool.copy_octahedra(slot)
    assert np.array_equal(dl, f["dl"]), f"{where}: {np.sum(dl != f['dl'])} DiagonalLength differ"


@pytest.mark.parametrize("seed", range(6))
def test_directional_random(lib, tmp_path, seed):
    inp = random_c(1000 + seed, str(tmp_path))
    p = ex.Problem.from_file(inp)
    o = Oracle(inp)
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    slot = pool.admit(p, device_check=False)
    compare(pool, slot, o, "after init")
    done = 0
    for n in (1, 7, 50, 300):
        pool.step(n)
        o.step(n)
        done += n
        compare(pool, slot, o, f"cycle {done}")
    pool.close()


@pytest.mark.parametrize("seed", range(4))
def test_directional_random_to_termination(lib, tmp_path, seed):
    inp = random_c(2000 + seed, str(tmp_path))
    p = ex.Problem.from_file(inp)
    o = Oracle(inp)
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    slot = pool.admit(p, device_check=False)
    assert pool.run_plain(slot) == o.run()
    compare(pool, slot, o, "final")
    pool.close()


@pytest.mark.parametrize("seed", range(4))
def test_spot_melt_random_to_termination(lib, tmp_path, seed):
    inp = random_s(3000 + seed, str(tmp_path))
    p = ex.Problem.from_file(inp)
    o = Oracle(inp)
    pool = ex.Pool(0, list_capacity=p.geometry.active_size)
    slot = pool.admit(p, device_check=False)
    compare(pool, slot, o, "after init")
    assert pool.run_plain(slot) == o.run()
    compare(pool, slot, o, "final")
    pool.close()


@pytest.mark.parametrize("seed", range(4))
def test_spot_melt_multilayer_random_to_termination(lib, tmp_path, seed):
    inp = random_s(4000 + seed, str(tmp_path), multilayer=True)
    p = ex.Problem.from_file(inp)
    o = Oracle(inp)
    pool = ex.Pool(0, list_capacity=p.geometry.domain_size)
    slot = pool.admit(p, device_check=False)
    compare(pool, slot, o, "after init")
    assert pool.run_plain(slot) == o.run()
    st = pool.status(slot)
    assert st.layer == int(open(inp).read().split("Number of layers:")[1].split()[0]) - 1
    o.fields()  # refreshes the oracle's window geometry
    assert (st.window_nz, st.window_nz * p.geometry.mx * p.geometry.my) == (o.nz_active, o.na)
    compare(pool, slot, o, "final")
    pool.close()


@pytest.mark.parametrize("seed", range(10))
def test_temperature_files_random_to_termination(lib, tmp_path, seed):
    inp = random_r(5000 + seed, str(tmp_path))
    p = ex.Problem.from_file(inp)
    o = Oracle(inp)
    pool = ex.Pool(0, list_capacity=p.geometry.domain_size)
    slot = pool.admit(p, device_check=False)
    compare(pool, slot, o, "after init")
    assert pool.run_plain(slot) == o.run()
    o.fields()
    compare(pool, slot, o, "final")
    pool.close()


def test_multilayer_needs_plain_path(lib, tmp_path):
    # the layer change runs between launches, so device-side termination is refused
    p = ex.Problem.from_file(random_s(4100, str(tmp_path), multilayer=True))
    pool = ex.Pool(0, list_capacity=p.geometry.domain_size)
    with pytest.raises(ex.ExacaError) as e:
        pool.admit(p, device_check=True)
    assert e.value.code == -2
    pool.close()
