"""Grain statistics of a final GrainID field: a numpy restatement of the reference analysis
(analysis/src/GAprint.cpp:17-198, PrintMisorientationData and PrintSizeData) over one
representative region. Test infrastructure: the checker of the device implementation and of the
statistical agreement with the reference's OpenMP build; nothing in the product imports it.

Fields are the solver's rank-local arrays (index k*mx*my + i*my + j with the ghost ring, mx = nx + 2,
my = ny + 2); the region is in the coordinates of the reference's .vtk output (k, i, j in
[0, nz) x [0, nx) x [0, ny)), default the interior without the wall layers.
"""
import math

import numpy as np

NUM_ORIENTATIONS = 10000
HIST_BINS = 64


def misorientation_table(guv: np.ndarray) -> np.ndarray:
    """Per orientation: the smallest angle (degrees) between the +Z axis and the three unit vectors,
    starting from 62.7 (GAprint.cpp:38-46)."""
    g = np.asarray(guv, dtype=np.float32).reshape(-1, 3, 3)
    out = np.empty(len(g), dtype=np.float32)
    for n in range(len(g)):
        amin = 62.7
        for ll in range(3):
            a = abs((180 / math.pi) * math.acos(float(g[n, ll, 2])))
            if a < amin:
                amin = a
        out[n] = amin
    return out


def region_view(field: np.ndarray, nx: int, ny: int, nz: int, region=None) -> np.ndarray:
    """The region of a rank-local field as an array (k, i, j)."""
    mx, my = nx + 2, ny + 2
    f = np.asarray(field).reshape(nz, mx, my)[:, 1:nx + 1, 1:ny + 1]
    xmin, xmax, ymin, ymax, zmin, zmax = region or (1, nx - 2, 1, ny - 2, 1, nz - 2)
    return f[zmin:zmax + 1, xmin:xmax + 1, ymin:ymax + 1]


def grain_stats(grain_id, melted, guv, nx, ny, nz, deltax, region=None) -> dict:
    gid = region_view(grain_id, nx, ny, nz, region).astype(np.int64)
    mel = region_view(melted, nx, ny, nz, region)
    table = misorientation_table(guv)
    ori = (np.abs(gid) - 1) % NUM_ORIENTATIONS
    mis = table[ori]
    m = mel == 1
    vol = gid.size
    n_grains = len(np.unique(gid))
    top = m[-1]
    hist = np.bincount(np.minimum(mis[m].astype(np.int64), HIST_BINS - 1), minlength=HIST_BINS)
    return dict(
        region_cells=int(vol), melted_cells=int(m.sum()), n_grains=int(n_grains),
        mean_grain_volume_um3=deltax * deltax * 1e12 * (vol / n_grains),
        nucleated_fraction=float((gid < 0).sum()) / vol,
        mean_misorientation_deg=float(mis[m].astype(np.float64).sum() / max(m.sum(), 1)),
        mean_misorientation_top_deg=float(mis[-1][top].astype(np.float64).sum() / max(top.sum(), 1)),
        misorientation_hist=hist.tolist(),
    )


def agree(a: dict, b: dict, tol: float = 0.02) -> dict:
    """Relative differences of grain count, mean grain volume, mean misorientation, and the total
    variation distance of the normalised misorientation histograms; 'ok' when all are within tol."""
    def rel(x, y):
        return abs(x - y) / max(abs(y), 1e-30)

    pa = np.array(a["misorientation_hist"], float)
    pb = np.array(b["misorientation_hist"], float)
    tv = 0.5 * np.abs(pa / pa.sum() - pb / pb.sum()).sum()
    d = dict(n_grains=rel(a["n_grains"], b["n_grains"]),
             mean_grain_volume=rel(a["mean_grain_volume_um3"], b["mean_grain_volume_um3"]),
             mean_misorientation=rel(a["mean_misorientation_deg"], b["mean_misorientation_deg"]),
             histogram_tv=float(tv))
    d["ok"] = all(v <= tol for v in d.values())
    return d
