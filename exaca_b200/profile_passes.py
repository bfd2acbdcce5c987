"""Per-pass timing of the directional-solidification case (G = R = 1e6, N = 25, 1e14 m^-3 nuclei,
2 % active substrate): admits an n^3 domain, runs `--warm` cycles in the persistent kernel, then
`--cycles` cycles as separate pass kernels (k_step_begin, k_grow, k_claim, k_capture_pass) and
prints their summed CUDA-event times. Under ncu this isolates one pass kernel on a front that has
had time to form:

    python -m exaca_b200.profile_passes 256 --warm 3000 --cycles 3
    python -m exaca_b200.profile_passes 288 --warm 4000 --launch 1000   # four k_cycles launches
    python -m exaca_b200.profile_passes 288 --warm 4000 --launch 1000 --config 0   # 4 lanes, 2 records
    ncu --set full --clock-control none -k regex:k_grow -s 1 -c 1 -o prof_grow256 \\
        python -m exaca_b200.profile_passes 256 --warm 3000 --cycles 3
"""
import argparse
import json

import exaca_b200 as ex

# the bench's workload (bench.py: WORKLOAD)
WORKLOAD = dict(G=1e6, R=1e6, n_ratio=25, nucleation_density=100.0, dTN=3.0, dTsigma=0.5, fract_surface_active=0.02)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("size", type=int, nargs="?", default=256, help="cube side in cells")
    ap.add_argument("--warm", type=int, default=3000, help="cycles in the persistent kernel first")
    ap.add_argument("--launch", type=int, default=0,
                    help="cycles per persistent launch of the warm-up (0: one launch), so a profiler can pick one")
    ap.add_argument("--cycles", type=int, default=3, help="cycles as separate pass kernels")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--config", type=int, default=-1,
                    help="step configuration (exaca_pool_set_config; -1: the pool's default)")
    args = ap.parse_args()
    n = args.size
    prob = ex.Problem.directional(n, n, n, **WORKLOAD)
    pool = ex.Pool(args.device, list_capacity=prob.geometry.active_size)
    try:
        if args.config >= 0:
            pool.set_config(args.config)
        pool.admit(prob, device_check=False)
        if args.launch > 0:
            done = 0
            while done < args.warm:
                pool.step(min(args.launch, args.warm - done))
                done += args.launch
        else:
            pool.step(args.warm)
        passes = pool.profile_cycles(args.cycles)
        print(json.dumps({"size": n, "warm_cycles": args.warm, "pass_cycles": args.cycles,
                          "ms_per_pass": passes}), flush=True)
    finally:
        pool.close()


if __name__ == "__main__":
    main()
