"""The host initialisation's random stream (exaca_b200/csrc/rng.hpp, rng.cpp) against libstdc++'s own
std::mt19937_64 and std::uniform_real_distribution<double>(0, 1), which the reference draws from
(src/CAinitialize.cpp:1464-1465, 1603-1604, 1844-1845): the same outputs and the same doubles, and
the threshold scan finds exactly the draws a per-draw comparison finds. No GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "exaca_b200", "csrc")

DRIVER = r"""
#include "rng.hpp"
#include <cstdio>
#include <random>
int main() {
    long bad = 0;
    for (unsigned long long seed : {0ull, 1ull, 987654321ull}) {
        std::mt19937_64 a(seed), a2(seed);
        std::uniform_real_distribution<double> dis(0.0, 1.0);
        exaca::Mt64 b(seed), b2(seed);
        for (long i = 0; i < 3000000; i++) {
            bad += a() != b.next();
            bad += dis(a2) != exaca::uniform01(b2.next());
        }
    }
    // the largest outputs: the draw that rounds up to 1 becomes the largest double below 1
    std::printf("clamp %d\n", exaca::uniform01(~0ull) == 0x1.fffffffffffffp-1);
    for (double p : {1e-4, 2e-2, 0.08, 0.5, 3.7e-9}) {
        std::mt19937_64 a(0);
        std::uniform_real_distribution<double> dis(0.0, 1.0);
        exaca::Mt64 b(0);
        const unsigned long long lim = exaca::uniform01_limit(p);
        long n_a = 0, n_b = 0, s_a = 0, s_b = 0;
        for (long i = 0; i < 2000003; i++)
            if (dis(a) < p) { n_a++; s_a += i; }
        // in uneven pieces, so that scans start and end inside the 312-output blocks
        long base = 0;
        for (long piece : {1L, 311L, 312L, 1000L, 1998379L}) {
            b.scan_below(piece, lim, [&](unsigned long long t) { n_b++; s_b += base + (long)t; });
            base += piece;
        }
        bad += n_a != n_b || s_a != s_b;
        std::printf("p %g draws below %ld %ld\n", p, n_a, n_b);
    }
    std::printf("mismatches %ld\n", bad);
    return bad != 0;
}
"""


def test_stream_equals_libstdcxx(tmp_path):
    src = tmp_path / "rng_driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "rng_driver"
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, str(src), os.path.join(CSRC, "rng.cpp"), "-o",
                        str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0" in out.stdout and "clamp 1" in out.stdout
