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
