"""C ABI surface and host-side behaviour of the native library, without a GPU: every function the
header declares is exported, problems are built and described on the host, and malformed inputs
fail with the reference's messages (src/CAinitialize.cpp:36-229) as error codes, not exceptions."""
import os
import re

import numpy as np
import pytest

from helpers import input_path, reference_error

import exaca_b200 as ex

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "exaca_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(exaca_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding covers the whole header
    assert set(names) == set(ex.SIGNATURES)


def test_problem_geometry_on_host(lib):
    p = ex.Problem.from_file(input_path("DirS64"))
    g = p.geometry
    # "64^3" type-C problem: nx = 64 + 2 walls, plus the ghost ring of the one-rank decomposition
    assert (g.nx, g.ny, g.nz, g.mx, g.my) == (66, 66, 66, 68, 68)
    assert g.domain_size == 68 * 68 * 66 and g.active_size == g.domain_size
    assert g.simulation_type == b"C"
    s = ex.Problem.from_file(input_path("SmallSpotMelt"))
    # spot melt: nz = R + 3, nx = 4 + 2R + offset (nspots - 1) (src/CAinitialize.cpp:508-510)
    assert (s.geometry.nx, s.geometry.ny, s.geometry.nz, s.geometry.nz_active) == (54, 79, 28, 27)


def test_directional_params_equal_input_file(lib, tmp_path):
    # the synthetic constructor and the equivalent input file give the same initial fields
    text = open(input_path("DirSNuc")).read()
    a = ex.Problem.from_file(input_path("DirSNuc")).fields()
    b = ex.Problem.directional(40, 47, 36, G=1e6, R=1e6, n_ratio=25, nucleation_density=2000, dTN=3.0,
                               dTsigma=0.5, fract_surface_active=0.02).fields()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def write(tmp_path, name, lines):
    p = tmp_path / name
    p.write_text("\n".join(lines) + "\n")
    return str(p)


BASE = open(os.path.join(ROOT, "tests", "golden", "inputs", "SmallDirS.txt")).read().splitlines()


def variant(replace=None, drop=None):
    out = []
    for ln in BASE:
        if drop and ln.startswith(drop):
            continue
        if replace:
            for k, v in replace.items():
                if ln.startswith(k):
                    ln = v
        out.append(ln)
    return out


@pytest.mark.parametrize(
    "lines,code,msg",
    [
        (variant(replace={"Problem type": "Problem type C"}), -1, 'must be separated from value by ":"'),
        (variant(drop="Cell size"), -1, 'Required input not present: "Cell size"'),
        (variant(replace={"Material": "Material: NoSuchAlloy"}), -1, "Could not locate/open Materials file"),
        (variant(replace={"Print Paraview vtk file of grain misorientation": "Print Paraview vtk file of grain misorientation values (Y or N)?: maybe"}), -1, 'must be "Y" or "N"'),
        (variant(replace={"Domain size in x": "Domain size in x: forty"}), -1, "invalid number"),
        (variant(replace={"Problem type": "Problem type: R"}), -1, None),
    ],
)
def test_malformed_inputs(lib, tmp_path, lines, code, msg):
    path = write(tmp_path, "bad.txt", lines)
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(path)
    assert e.value.code == code
    if msg:
        assert msg in str(e.value)
    # the reference itself (where built here) stops on the same file with the same message
    ref = reference_error(str(path))
    assert ref is None or (ref and ref in str(e.value)), (ref, str(e.value))


def test_multilayer_problem_and_layer_limit(lib, tmp_path):
    lines = open(input_path("SmallSpotMelt")).read().splitlines()
    two = [("Number of layers: 2" if l.startswith("Number of layers") else l) for l in lines]
    p = ex.Problem.from_file(write(tmp_path, "ml.txt", two))
    assert p.geometry.nz > p.geometry.nz_active
    # LayerID is kept in 8 bits on the device
    many = [("Number of layers: 200" if l.startswith("Number of layers") else l) for l in lines]
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(write(tmp_path, "ml200.txt", many))
    assert e.value.code == -2
    assert "between 1 and 127" in str(e.value)


def test_missing_input_file(lib):
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file("/nonexistent/input.txt")
    assert "Could not locate/open Input file" in str(e.value)


def test_null_arguments_return_codes(lib):
    assert lib.exaca_problem_from_file(None, None) == -5
    assert lib.exaca_pool_step(None, 1) == -5
    assert lib.exaca_pool_status(None, 0, None) == -5
    assert lib.exaca_problem_slot_bytes(None) == -1
