"""Pin the 512^3 directional-solidification solve (the benchmark workload) without dense fixtures.

Writes tests/golden/DirS512.json: SHA-256 digests of GrainID (int32) and CellType (int8) over the
whole 516 x 516 x 514 cell array, at two points of the solve:

  cycle5000   after 5000 cycles, from the UNMODIFIED reference (Serial dispatch, the project's
              shims; oracle/_ref/ref_bench_serial runs the reference's own initialisation and step
              functions in RunProgram_Reduced's order) and from the restatement (oracle/_port):
              both must agree. The reference's 32-bit `26 * D3D1ConvPosition` (src/CAupdate.cpp:336)
              overflows once active cells lie above z ~ 310, which the solve reaches near cycle
              7700, so a complete reference run is not possible at this size; 5000 cycles are
              below that.
  final       at termination, from the restatement (64-bit indices throughout), with the final
              cycle and the census lines the reference prints every 1000 cycles.

The input is bench.py's 512^3 input file, so the benchmark's own solve can be checked against it.
Needs the reference sources (build container only) for the `ref` stage; run stages separately with
`--stage ref` / `--stage port` (each merges its keys into the JSON). Takes hours on one host.

    python tests/golden/make_dirs512.py [--stage ref|port|all] [--threads T] [--size N]
"""
import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from bench import input_file_text  # noqa: E402

REF_SERIAL = os.path.join(ROOT, "oracle", "_ref", "ref_bench_serial")
PIN_CYCLE = 5000


def digests(grain_id, cell_type):
    return {
        "sha_grain_id": hashlib.sha256(np.ascontiguousarray(grain_id, dtype=np.int32).tobytes()).hexdigest(),
        "sha_cell_type": hashlib.sha256(np.ascontiguousarray(cell_type).astype(np.int8).tobytes()).hexdigest(),
    }


def stage_ref(inp, work, pin_cycle):
    if not os.path.exists(REF_SERIAL):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "-j8"], check=True)
    dump = os.path.join(work, "ref_dump.bin")
    t0 = time.time()
    r = subprocess.run([REF_SERIAL, inp, str(pin_cycle // 1000), "1000", dump], cwd=work, capture_output=True,
                       text=True, check=True)
    a = np.fromfile(dump, np.int32)
    n = a.size // 2
    os.remove(dump)
    # a census line may follow text the reference printed without a line break
    census = [m.group(0) for m in re.finditer(r"cycle = \d+ Superheated.*|^Jumping to cycle \d+", r.stdout,
                                              re.MULTILINE)]
    out = digests(a[:n], a[n:])
    out.update(cells=int(n), census=census, seconds=round(time.time() - t0, 1))
    return out


def stage_port(inp, pin_cycle, threads):
    from oracle_port import Oracle

    Oracle.set_threads(threads)
    t0 = time.time()
    o = Oracle(inp)
    paused = o.run_to(pin_cycle)
    assert paused, "the solve ended before the pinned cycle"
    f = o.fields()
    at_pin = digests(f["grain_id"], f["cell_type"])
    at_pin["census"] = o.census_lines()
    del f
    t1 = time.time()
    final_cycle = o.run()
    f = o.fields()
    final = digests(f["grain_id"], f["cell_type"])
    final.update(cycle=int(final_cycle), census=o.census_lines(), cells=int(f["grain_id"].size))
    at_pin["seconds"] = round(t1 - t0, 1)
    final["seconds"] = round(time.time() - t0, 1)
    return at_pin, final


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", choices=["ref", "port", "all"], default="all")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    name = "DirS512" if args.size == 512 else f"DirS{args.size}"
    out_path = args.out or os.path.join(HERE, name + ".json")
    doc = json.load(open(out_path)) if os.path.exists(out_path) else {}
    doc["input"] = input_file_text(args.size).splitlines()
    doc["pin_cycle"] = PIN_CYCLE
    work = tempfile.mkdtemp(prefix="dirs512_")
    inp = os.path.join(work, "input.txt")
    with open(inp, "w") as fh:
        fh.write(input_file_text(args.size))
    if args.stage in ("ref", "all"):
        doc["cycle5000_reference"] = stage_ref(inp, work, PIN_CYCLE)
        json.dump(doc, open(out_path, "w"), indent=1)
        print("reference at cycle", PIN_CYCLE, doc["cycle5000_reference"]["sha_grain_id"], flush=True)
    if args.stage in ("port", "all"):
        doc["cycle5000_restatement"], doc["final"] = stage_port(inp, PIN_CYCLE, args.threads)
        json.dump(doc, open(out_path, "w"), indent=1)
        print("restatement: final cycle", doc["final"]["cycle"], flush=True)
    for k in ("sha_grain_id", "sha_cell_type"):
        a = doc.get("cycle5000_reference", {}).get(k)
        b = doc.get("cycle5000_restatement", {}).get(k)
        if a and b and a != b:
            raise SystemExit(f"reference and restatement differ at cycle {PIN_CYCLE} ({k})")
    os.rmdir(work) if not os.listdir(work) else None


if __name__ == "__main__":
    main()
