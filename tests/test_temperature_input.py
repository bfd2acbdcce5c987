"""Type-R input errors on the host (no GPU): the reference's messages for a temperature-file
header with a wrong column (src/CAinitialize.cpp:149-175), the old header format (:763-775) and a
temperature grid that is not a whole multiple of the cell size (:1140-1152) and a missing
temperature file (:201-209), plus the solver's own
limit on distinct UndercoolingChange values (one growth table each). Each case is the RTrackH2
golden problem with one change. Where the reference compiled against single-rank shims is present
(oracle/_ref), it runs on the same files and must raise the same message (or none)."""
import os

import pytest
from helpers import reference_error

import exaca_b200 as ex

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INPUTS = os.path.join(ROOT, "tests", "golden", "inputs")
TRACK = os.path.join(INPUTS, "temperatures", "track_h2.csv")
def r_case(tmp_path, header=None, first_line=None, mesh=None, rate=None):
    """RTrackH2 with its temperature file copied to tmp_path and changed as asked."""
    rows = open(TRACK).read().splitlines()
    if header is not None:
        rows[0] = header
    if rate is not None:
        rows = [rows[0]] + [",".join(r.split(",")[:5] + [repr(rate(i))]) for i, r in enumerate(rows[1:])]
    if first_line is not None:
        rows.insert(0, first_line)
    tdir = tmp_path / "temperatures"
    tdir.mkdir()
    (tdir / "track_h2.csv").write_text("\n".join(rows) + "\n")
    out = []
    for ln in open(os.path.join(INPUTS, "RTrackH2.txt")).read().splitlines():
        if ln.startswith("Path to temperature file"):
            ln = f"Path to temperature file(s): {tdir}"
        elif mesh is not None and ln.startswith("Heat transport data mesh size"):
            ln = f"Heat transport data mesh size (microns): {mesh}"
        out.append(ln)
    path = tmp_path / "in.txt"
    path.write_text("\n".join(out) + "\n")
    return str(path)


def test_unchanged_copy_initialises(lib, tmp_path):
    prob = ex.Problem.from_file(r_case(tmp_path))
    assert prob.geometry.active_size > 0


@pytest.mark.parametrize(
    "header,msg",
    [
        ("x,y,z,tm,tl,rate", "cr not found in temperature file header"),
        ("x,y,z,tm,tliq,cr", "ts not found in temperature file header"),
        ("X, Y ,Z,TM,Ts,R", None),  # case and blanks do not matter, and the alternative names are accepted
    ],
)
def test_temperature_header(lib, tmp_path, header, msg):
    path = r_case(tmp_path, header=header)
    ref = reference_error(path)
    if msg is None:
        ex.Problem.from_file(path)
        assert ref in (None, "")
        return
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(path)
    assert e.value.code == -1 and msg in str(e.value)
    assert ref in (None, msg)


def test_old_temperature_format(lib, tmp_path):
    path = r_case(tmp_path, first_line="Number of temperature data points: 667")
    msg = "Error: Old header and temperature file format no longer supported"
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(path)
    assert e.value.code == -1 and msg in str(e.value)
    assert reference_error(path) in (None, msg)


def test_temperature_spacing_not_a_multiple_of_the_cell_size(lib, tmp_path):
    path = r_case(tmp_path, mesh=2.5)
    msg = "Error: Temperature data point spacing not evenly divisible by CA cell size"
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(path)
    assert e.value.code == -1 and msg in str(e.value)
    assert reference_error(path) in (None, msg)


def test_too_many_undercooling_values(lib, tmp_path):
    # a cooling rate of its own for every temperature point: interpolated onto the 1 um cells, the
    # melted cells get far more than 1024 distinct UndercoolingChange values
    path = r_case(tmp_path, rate=lambda i: 1.0e5 + 997.0 * i)
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(path)
    assert e.value.code == -2 and "distinct UndercoolingChange values" in str(e.value)


def test_missing_temperature_file(lib, tmp_path):
    # one file in the series: its name carries no number, and only numbered files exist here
    lines = []
    for ln in open(os.path.join(INPUTS, "RTwoFiles3Layers.txt")).read().splitlines():
        if ln.startswith("Number of temperature files"):
            ln = "Number of temperature files: 1"
        elif ln.startswith("Path to temperature file"):
            ln = "Path to temperature file(s): " + os.path.join(INPUTS, "temperatures")
        lines.append(ln)
    path = tmp_path / "in.txt"
    path.write_text("\n".join(lines) + "\n")
    msg = "Could not locate/open Temperature file"
    with pytest.raises(ex.ExacaError) as e:
        ex.Problem.from_file(str(path))
    assert e.value.code == -1 and msg in str(e.value)
    assert reference_error(str(path)) in (None, msg)
