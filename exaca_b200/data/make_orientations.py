"""Write the orientation table shipped with this package.

10,000 rotation matrices drawn uniformly from SO(3) (Shoemake's unit-quaternion method, K. Shoemake,
"Uniform random rotations", Graphics Gems III, 1992) from a fixed NumPy PCG64 seed. Each line holds
the three rows of one matrix as 9 comma-separated values with 6 significant digits, after a first
line giving the count: the layout the ExaCA input key "File of grain orientations" expects
(reader: src/CAinitialize.cpp:1408-1441 of the reference).

Usage: python make_orientations.py [out.csv]
"""
import sys

import numpy as np

N = 10000
SEED = 20211203


def rotations(n: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.random((n, 3))
    q = np.stack(
        [
            np.sqrt(1 - u[:, 0]) * np.sin(2 * np.pi * u[:, 1]),
            np.sqrt(1 - u[:, 0]) * np.cos(2 * np.pi * u[:, 1]),
            np.sqrt(u[:, 0]) * np.sin(2 * np.pi * u[:, 2]),
            np.sqrt(u[:, 0]) * np.cos(2 * np.pi * u[:, 2]),
        ],
        axis=1,
    )
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - z * w)
    r[:, 0, 2] = 2 * (x * z + y * w)
    r[:, 1, 0] = 2 * (x * y + z * w)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - x * w)
    r[:, 2, 0] = 2 * (x * z - y * w)
    r[:, 2, 1] = 2 * (y * z + x * w)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r.reshape(n, 9)


def main() -> None:
    out = sys.argv[1] if len(sys.argv) > 1 else "Substrate/GrainOrientationVectors_Uniform10k.csv"
    r = rotations(N, SEED)
    with open(out, "w") as f:
        f.write(f"{N}\n")
        for row in r:
            f.write(",".join(f"{v:.6g}" for v in row) + "\n")


if __name__ == "__main__":
    main()
