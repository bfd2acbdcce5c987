"""Seeded random ExaCA input files for the oracle-vs-GPU parity tests (test infrastructure)."""
import os

import numpy as np

C_TEMPLATE = """Random directional-solidification parity case {name}
*****
Problem type: C
Decomposition strategy: 1
Material: Inconel625
Cell size (microns): 1
Heterogeneous nucleation density (normalized by 1*10^12 per m^3): {density}
Mean nucleation undercooling (in K): {dtn}
Standard deviation of nucleation undercooling: {sigma}
Path to output: {out}/
Output file base name: {name}
File of grain orientations: GrainOrientationVectors_Uniform10k.csv
Thermal gradient (K/m): {G}
Cooling rate (K/s): {R}
Domain size in x: {nx}
Domain size in y: {ny}
Domain size in z: {nz}
"N", where the time step = deltax/(Steady State Velocity * N): {N}
Fraction of surface sites active: {frac}
***Output data printing options: (Y or N) which data should be printed***
Print Paraview vtk file of grain misorientation values (Y or N)?: N
Print Paraview vtk file of all ExaCA data for post-processing (Y or N)?: N
Debug check (reduced)- Print data for main Kokkos views (CellType, LayerID, CritTimeStep) following initialization for debug check (Y or N)?: N
Debug check (extensive) - Print data for all main data structures (CellType, GrainID, CritTimeStep, UndercoolingCurrent, UndercoolingChange, Melted, LayerID) following initialization for debug check (Y or N)?: N
"""

S_TEMPLATE = """Random spot-melt parity case {name}
*****
Problem type: S
Decomposition strategy: 1
Material: Inconel625
Cell size (microns): 1
Heterogeneous nucleation density (normalized by 1*10^12 per m^3): {density}
Mean nucleation undercooling (in K): {dtn}
Standard deviation of nucleation undercooling: {sigma}
Path to output: {out}/
Output file base name: {name}
File of grain orientations: GrainOrientationVectors_Uniform10k.csv
Thermal gradient (K/m): {G}
Cooling rate (K/s): {R}
Number of spots in x: {sx}
Number of spots in y: {sy}
Offset between spot centers (in microns): {off}
Radii of spots (in microns): {rad}
Number of layers: {layers}
Offset between layers (in cells): {lh}
"N", where the time step = deltax/(Steady State Velocity * N): {N}
Substrate grain spacing (in microns): {spacing}
***Output data printing options: (Y or N) which data should be printed***
Print Paraview vtk file of grain misorientation values (Y or N)?: N
Print Paraview vtk file of all ExaCA data for post-processing (Y or N)?: N
Debug check (reduced)- Print data for main Kokkos views (CellType, LayerID, CritTimeStep) following initialization for debug check (Y or N)?: N
Debug check (extensive) - Print data for all main data structures (CellType, GrainID, CritTimeStep, UndercoolingCurrent, UndercoolingChange, Melted, LayerID) following initialization for debug check (Y or N)?: N
"""


R_TEMPLATE = """Random temperature-file parity case {name}
*****
Problem type: R
Decomposition strategy: 1
Material: Inconel625
Cell size (microns): 1
Heterogeneous nucleation density (normalized by 1*10^12 per m^3): {density}
Mean nucleation undercooling (in K): {dtn}
Standard deviation of nucleation undercooling: {sigma}
Path to output: {out}/
Output file base name: {name}
File of grain orientations: GrainOrientationVectors_Uniform10k.csv
Heat transport data mesh size (microns): {h}
Time step (microseconds): {dt}
Substrate grain spacing (in microns): {spacing}
Path to temperature file(s): {out}
Temperature filename (* glob before the name): {tname}
Number of temperature files: {nfiles}
Extra set of wall cells around temperature field (used for spot melt problems, Y or N)?: N
Number of layers: {layers}
Offset between layers (if Number of layers > 1, in cells): {lh}
***Output data printing options: (Y or N) which data should be printed***
Print Paraview vtk file of grain misorientation values (Y or N)?: N
Print Paraview vtk file of all ExaCA data for post-processing (Y or N)?: N
Debug check (reduced)- Print data for main Kokkos views (CellType, LayerID, CritTimeStep) following initialization for debug check (Y or N)?: N
Debug check (extensive) - Print data for all main data structures (CellType, GrainID, CritTimeStep, UndercoolingCurrent, UndercoolingChange, Melted, LayerID) following initialization for debug check (Y or N)?: N
"""


def random_r(seed, outdir):
    """Seeded random type-R input with its temperature files (1 or 2 in series, 1-3 layers, a 1 or
    2 um temperature grid): half-ellipsoid melt tracks along x, two cooling rates by depth."""
    r = np.random.default_rng(seed)
    name = f"rr{seed}"
    h_um = int(r.integers(1, 3))
    h = h_um * 1e-6
    nfiles = int(r.integers(1, 3))
    tname = f"{name}.csv"
    for f in range(nfiles):
        nxp, nyp, nzp = int(r.integers(8, 20)), int(r.integers(6, 12)), int(r.integers(3, 6))
        width, depth = (0.3 + 0.2 * r.random()) * nyp * h, (0.6 + 0.3 * r.random()) * (nzp - 1) * h
        v = float(10 ** r.uniform(-0.5, 0.3))
        cr = (float(10 ** r.uniform(5.5, 6.2)), float(10 ** r.uniform(5.2, 5.9)))
        rows = ["x,y,z,tm,tl,cr"]
        yc = 0.5 * (nyp - 1) * h
        for i in range(nxp):
            for j in range(nyp):
                for k in range(nzp):
                    x, y, z = i * h, j * h, -k * h
                    if ((y - yc) / width) ** 2 + (z / max(depth, h)) ** 2 > 1.0:
                        continue
                    tl = x / v + 2e-6 * k * h / max(depth, h) + 1e-7 * r.random() + 2e-6
                    c = cr[0] if k * h < 0.5 * depth else cr[1]
                    if r.random() < 0.05:
                        rows.append(",".join(repr(float(q)) for q in (x, y, z, tl - 1e-5, tl - 5e-6, 0.5 * c)))
                    rows.append(",".join(repr(float(q)) for q in (x, y, z, tl - 5e-6, tl, c)))
        fname = (f"{f + 1}" if nfiles > 1 else "") + tname
        open(os.path.join(outdir, fname), "w").write("\n".join(rows) + "\n")
    txt = R_TEMPLATE.format(
        name=name, out=outdir, h=h_um, dt=round(float(r.uniform(0.03, 0.08)), 3),
        density=round(float(10 ** r.uniform(0, 2.7)), 3), dtn=round(float(r.uniform(1, 6)), 2),
        sigma=round(float(r.uniform(0.2, 1.0)), 2), spacing=round(float(r.uniform(3, 8)), 2), tname=tname,
        nfiles=nfiles, layers=int(r.integers(1, 4)), lh=int(r.integers(2, 5)))
    path = os.path.join(outdir, name + ".txt")
    open(path, "w").write(txt)
    return path


def random_c(seed, outdir):
    r = np.random.default_rng(seed)
    name = f"rc{seed}"
    txt = C_TEMPLATE.format(
        name=name, out=outdir, nx=int(r.integers(12, 41)), ny=int(r.integers(12, 41)), nz=int(r.integers(12, 41)),
        G=float(10 ** r.uniform(5, np.log10(5e6))), R=float(10 ** r.uniform(4, 6)),
        density=round(float(10 ** r.uniform(0, 3.3)), 3), dtn=round(float(r.uniform(1, 6)), 2),
        sigma=round(float(r.uniform(0.2, 1.0)), 2), N=int(r.integers(8, 31)), frac=round(float(r.uniform(0.005, 0.15)), 4))
    path = os.path.join(outdir, name + ".txt")
    open(path, "w").write(txt)
    return path


def random_s(seed, outdir, multilayer=False):
    """Seeded random spot-melt input; with multilayer, 2-4 layers 3 to R cells apart (drawn after
    the single-layer parameters, so those stay the same for a seed)."""
    r = np.random.default_rng(seed)
    name = f"rs{seed}"
    rad = int(r.integers(6, 13))
    prm = dict(
        name=name, out=outdir, sx=int(r.integers(1, 3)), sy=int(r.integers(1, 3)), rad=rad,
        off=int(r.integers(rad // 2, rad + 4)), G=float(10 ** r.uniform(5, 6.5)), R=float(10 ** r.uniform(5, 6.5)),
        density=round(float(10 ** r.uniform(0, 3)), 3), dtn=round(float(r.uniform(1, 6)), 2),
        sigma=round(float(r.uniform(0.2, 1.0)), 2), N=int(r.integers(10, 31)),
        spacing=round(float(r.uniform(4, 12)), 2), layers=1, lh=10)
    if multilayer:
        prm["layers"] = int(r.integers(2, 5))
        prm["lh"] = int(r.integers(3, rad + 1))
    txt = S_TEMPLATE.format(**prm)
    path = os.path.join(outdir, name + ".txt")
    open(path, "w").write(txt)
    return path
