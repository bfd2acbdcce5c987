"""Writes the synthetic temperature-data files of the type-R golden cases (test infrastructure).

The reference repository ships no temperature data (examples/Temperatures is not in it), so the
type-R parity cases read seeded synthetic files in the reference's reduced format
(src/CAinitialize.cpp:149-187): a header line "x,y,z,tm,tl,cr", then one comma-separated point per
line, coordinates in m, melting / liquidus times in s, cooling rate in K/s.

Each file is one pass of a heat source along +x over a rectangular region: a point (x, y, z) of the
heat-transport grid (spacing h) is melted when it lies inside the half-ellipsoidal track
((y - yc) / w)^2 + (z / d)^2 <= 1 (z <= 0 is depth below the top surface); its liquidus time is
x / v plus a depth lag, and its cooling rate takes one of two values (upper and lower part of the
track), so UndercoolingChange takes a few values after the reference's interpolation. Some points
are listed twice, the first time with an earlier liquidus time, which the reference must discard
("only keep the last time that this point went below the liquidus"). numpy default_rng seeds make
the files reproducible.

Usage: python tests/golden/make_temperatures.py   (rewrites tests/golden/inputs/temperatures/*.csv)
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "inputs", "temperatures")


def track(seed, nx_pts, ny_pts, nz_pts, h, v, width, depth, cr_top, cr_bottom, t0=0.0):
    rng = np.random.default_rng(seed)
    yc = 0.5 * (ny_pts - 1) * h
    rows = []
    for i in range(nx_pts):
        for j in range(ny_pts):
            for k in range(nz_pts):
                x, y, z = i * h, j * h, -k * h
                if ((y - yc) / width) ** 2 + (z / depth) ** 2 > 1.0:
                    continue
                lag = 2e-6 * (k * h) / depth + 1e-7 * rng.random()
                tl = t0 + x / v + lag
                tm = tl - 5e-6
                cr = cr_top if k * h < 0.5 * depth else cr_bottom
                if rng.random() < 0.05:
                    # an earlier pass below the liquidus, superseded by the later one
                    rows.append((x, y, z, tm - 1e-5, tl - 1e-5, 0.5 * cr))
                rows.append((x, y, z, tm, tl, cr))
    return rows


def write(name, rows):
    os.makedirs(OUT, exist_ok=True)
    with open(os.path.join(OUT, name), "w") as f:
        f.write("x,y,z,tm,tl,cr\n")
        for r in rows:
            f.write(",".join(repr(float(v)) for v in r) + "\n")


def main():
    # one track on a 2 um grid (the CA grid of 1 um interpolates between points)
    write("track_h2.csv", track(11, 21, 11, 5, 2e-6, 0.5, 9e-6, 7e-6, 8e5, 5e5))
    # two tracks on a 1 um grid for a 2-file series, shifted in y
    write("1track_h1.csv", track(12, 30, 16, 6, 1e-6, 0.6, 6e-6, 5e-6, 9e5, 6e5))
    write("2track_h1.csv", track(13, 30, 16, 6, 1e-6, 0.6, 5e-6, 5e-6, 7e5, 4e5, t0=2e-6))


if __name__ == "__main__":
    main()
