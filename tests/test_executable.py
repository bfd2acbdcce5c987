"""The drop-in contract of the ExaCA-B200 executable against the reference's `ExaCA-Kokkos <input>`
(src/main.cpp:15-47), run as a subprocess on every golden case:

* stdout: the census lines printed every 1000 cycles and the type-S/R jump lines
  (src/CAupdate.cpp:776-780, 815) equal the reference's, in order; so do the lines of every layer
  change (src/CAinitialize.cpp:2810-2830, src/runCA.cpp:376-405), timing masked;
* the .log file (src/CAprint.cpp:486-548) equals the reference's line by line, with only the input
  file's path and the timing values masked;
* the .vtk and _Misorientations.vtk files equal the reference's bytes.
"""
import hashlib
import os
import re
import subprocess

import pytest

from helpers import copy_input, golden_cases, load_golden, output_base

import exaca_b200 as ex

FLOAT = re.compile(r"[-+]?(?:\d+\.?\d*(?:e[-+]?\d+)?|inf|nan)")
LAYER_LINES = ("New domain bottom", "New domain top", "New active domain height", "Resize executed",
               "New layer setup", "New layer ghost nodes", "Time for layer number")


def census_lines(text):
    return [m.group(0) for m in re.finditer(r"cycle = \d+ Superheated.*|^Jumping to cycle \d+", text, re.MULTILINE)]


def masked_log(text):
    """The .log with the run's own input path and its timing values replaced by placeholders."""
    out = []
    for ln in text.splitlines():
        if ln.startswith("log file for a simulation run with input file "):
            ln = re.sub(r"input file \S+ ", "input file <input> ", ln)
        elif ln.startswith("This simulation took") or ln.startswith("Max/min rank time"):
            ln = FLOAT.sub("<t>", ln)
        out.append(ln)
    return out


def layer_lines(text):
    out = []
    for ln in text.splitlines():
        if ln.startswith(LAYER_LINES):
            if ln.startswith("Time for layer number"):
                ln = re.sub(r" was \S+ s,", " was <t> s,", ln)
            out.append(ln)
    return out


def test_masking_keeps_everything_but_timing():
    """The mask leaves every non-timing character of the reference's .log in place."""
    log = str(load_golden("SpotMelt3Layers")["log"])
    m = masked_log(log)
    assert len(m) == len(log.splitlines())
    assert m[1].startswith("This simulation took <t> seconds") and all("<t>" in ln for ln in m if ln.startswith("Max/min"))
    assert m[2] == "This simulation was type: S" and "Rank 0 contained 36 cells in x" in "\n".join(m)


@pytest.mark.gpu
@pytest.mark.parametrize("case", golden_cases())
def test_executable_matches_reference(lib, case, tmp_path):
    g = load_golden(case)
    inp = copy_input(case, str(tmp_path))
    r = subprocess.run([ex.EXE_PATH, inp], cwd=str(tmp_path), capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-2000:]
    assert census_lines(r.stdout) == [str(x) for x in g["census"]]
    assert layer_lines(r.stdout) == layer_lines(str(g["stdout"]))
    base = os.path.join(str(tmp_path), output_base(case))
    assert masked_log(open(base + ".log").read()) == masked_log(str(g["log"]))
    for suffix, key in ((".vtk", "sha_vtk"), ("_Misorientations.vtk", "sha_mis")):
        assert hashlib.sha256(open(base + suffix, "rb").read()).hexdigest() == str(g[key]), suffix
