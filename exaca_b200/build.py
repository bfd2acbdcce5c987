"""Build recipe of the native library and executable (sm_100a only).

    python -m exaca_b200.build        # or exaca_b200.build.build()

Produces, in-tree:
    exaca_b200/lib/libexaca_b200.so   host C++ (parser, init, output, C ABI) + CUDA kernels
    exaca_b200/lib/ExaCA-B200         drop-in executable for `ExaCA-Kokkos <input file>`

Host C++ is compiled with -ffp-contract=off and the device code with -fmad=false so that no
floating-point expression is contracted into a fused multiply-add: the solver reproduces the
reference's rounding step by step.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)

HOST_SOURCES = ["input.cpp", "init.cpp", "output.cpp", "capi.cpp", "rng.cpp"]
# per-file optimisation level (the random-stream refill is vectorised at -O3)
HOST_OPT = {"rng.cpp": "-O3"}
CUDA_SOURCES = ["device.cu", "census_scratch.cu"]
HEADERS = ["exaca_host.hpp", "pool.hpp", "rng.hpp", "directions.hpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = "g++"
HOST_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(verbose=False):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "exaca_b200.h")]
    objs = []
    for s in HOST_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OBJ, s + ".o")
        if _newer(obj, [src] + hdrs):
            flags = [HOST_OPT.get(s, f) if f == "-O2" else f for f in HOST_FLAGS]
            _run([CXX] + flags + ["-c", src, "-o", obj])
        objs.append(obj)
    for s in CUDA_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OBJ, s + ".o")
        if _newer(obj, [src] + hdrs):
            _run(
                [NVCC] + GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true",
                                    "-prec-sqrt=true", "-Xcompiler", "-fPIC,-ffp-contract=off",
                                    "-Xptxas", "-v" if verbose else "-O3", "-c", src, "-o", obj]
            )
        objs.append(obj)
    so = os.path.join(LIB, "libexaca_b200.so")
    if _newer(so, objs):
        _run([NVCC] + GENCODE + ["-shared", "-o", so] + objs + ["-lcudart", "-ldl"])
    exe = os.path.join(LIB, "ExaCA-B200")
    main = os.path.join(SRC, "main.cpp")
    if _newer(exe, [so, main]):
        _run([CXX, "-O2", "-std=c++17", main, "-o", exe, "-L" + LIB, "-lexaca_b200", "-Wl,-rpath,$ORIGIN"])
    return so


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
