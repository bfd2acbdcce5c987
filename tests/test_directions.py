"""The compile-time direction encodings the kernels read (exaca_b200/csrc/directions.hpp): per
direction its x / y / z component masks, its opposite and the capture pass's slot order (directions
by z, then x, then y), checked against the neighbour tables on the host."""
import os
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))

CHECK = r"""
#include <cstdio>
#include "directions.hpp"
using namespace exaca;
static unsigned field5(unsigned long long a, unsigned long long b, unsigned long long c, int i) {
    unsigned long long v = i < 12 ? a : (i < 24 ? b : c);
    int f = i < 12 ? i : (i < 24 ? i - 12 : i - 24);
    return (unsigned)(v >> (5 * f)) & 31u;
}
static int comp(unsigned p, unsigned m, int l) { return (int)((p >> l) & 1u) - (int)((m >> l) & 1u); }
int main() {
    int bad = 0, n = 0;
    for (int l = 0; l < 26; l++) {
        bad += comp(kDirXP, kDirXM, l) != kNeighborX[l];
        bad += comp(kDirYP, kDirYM, l) != kNeighborY[l];
        bad += comp(kDirZP, kDirZM, l) != kNeighborZ[l];
        int o = (int)field5(kOppA, kOppB, kOppC, l);
        bad += kNeighborX[o] != -kNeighborX[l] || kNeighborY[o] != -kNeighborY[l] || kNeighborZ[o] != -kNeighborZ[l];
    }
    for (int dz = -1; dz <= 1; dz++)
        for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++) {
                if (!dz && !dx && !dy)
                    continue;
                int l = (int)field5(kSlotA, kSlotB, kSlotC, n++);
                bad += kNeighborZ[l] != dz || kNeighborX[l] != dx || kNeighborY[l] != dy;
            }
    std::printf("%d\n", bad);
    return bad != 0;
}
"""


def test_direction_encodings(tmp_path):
    src = tmp_path / "check.cpp"
    src.write_text(CHECK)
    exe = tmp_path / "check"
    try:
        subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "exaca_b200", "csrc"), str(src), "-o", str(exe)],
                       check=True, capture_output=True, text=True)
    except FileNotFoundError:
        pytest.skip("no host C++ compiler")
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout
