// Host-side problem set-up for the B200 solver: geometry, temperature field, substrate, grain seeds,
// nuclei, and the lookup tables the device kernels use.
//
// The random streams are the reference's (libstdc++ mt19937_64 / uniform_real_distribution,
// default_random_engine / normal_distribution) drawn in the reference's loop orders, so the same
// input file yields the same seeds and nuclei. Everything that is a pure per-cell function of these
// (the fresh-octahedron state of initially active cells, the Voronoi baseplate) is finished on the
// device when the problem is admitted to a pool.
#include "exaca_host.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

namespace exaca {

const int kNeighborX[26] = {0, 1, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, 0, 1, -1, 0, 0, 1, -1, 1, -1};
const int kNeighborY[26] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};
const int kNeighborZ[26] = {0, 0, 0, 1, -1, 1, 1, -1, -1, 1, -1, 1, 1, -1, -1, 0, 0, 0, 0, 0, 1, -1, 1, 1, -1, -1};

void build_itlist(int it[9][26], int lens[9]) {
    // Case 0 keeps all 26; the others drop the neighbours that would leave the rank's x/y extent
    // (src/CAinitialize.cpp:676-745).
    auto keep = [](int c, int n) {
        int x = kNeighborX[n], y = kNeighborY[n];
        switch (c) {
        case 0: return true;
        case 1: return y != -1;
        case 2: return y != 1;
        case 3: return x != -1;
        case 4: return x != 1;
        case 5: return x != -1 && y != -1;
        case 6: return x != 1 && y != -1;
        case 7: return x != -1 && y != 1;
        default: return x != 1 && y != 1;
        }
    };
    for (int c = 0; c < 9; c++) {
        int pos = 0;
        for (int n = 0; n < 26; n++) {
            it[c][n] = 0;
            if (keep(c, n))
                it[c][pos++] = n;
        }
        lens[c] = pos;
    }
}

void read_orientations(const std::string &path, std::vector<float> &guv) {
    // src/CAinitialize.cpp:1408-1441: skip the count line, then up to 10000 lines of 9 values
    guv.assign(9 * kNumOrientations, 0.0f);
    std::ifstream in(path);
    std::string line;
    std::getline(in, line);
    for (int i = 0; i < kNumOrientations; i++) {
        if (!std::getline(in, line))
            break;
        std::istringstream ss(line);
        int comp = 0, uv = 0;
        std::string tok;
        while (ss) {
            if (!std::getline(ss, tok, ','))
                break;
            float v = atof(tok.c_str());
            long idx = 9L * i + 3 * uv + comp;
            if (idx < 9L * kNumOrientations && uv < 3)
                guv[idx] = v;
            comp++;
            if (comp > 2) {
                comp = 0;
                uv++;
            }
        }
    }
}

// Critical diagonal lengths of a fresh octahedron (centre at the cell centre) for each orientation
// and each neighbour direction. Same expression and operation order as the reference's nucleation
// and grain-init code (src/CAupdate.cpp:112-194, src/CAinitialize.cpp:1963-2042), evaluated with
// the host libm so pow(., 0.5) rounds exactly as it does there.
void build_cdl_table(const std::vector<float> &guv, std::vector<float> &table) {
    table.assign(26L * kNumOrientations, 0.0f);
    for (int o = 0; o < kNumOrientations; o++) {
        const float *g = &guv[9L * o];
        for (int n = 0; n < 26; n++) {
            double x0 = kNeighborX[n];
            double y0 = kNeighborY[n];
            double z0 = kNeighborZ[n];
            double mag0 = pow(pow(x0, 2.0) + pow(y0, 2.0) + pow(z0, 2.0), 0.5);
            double d1x, d1y, d1z, d2x, d2y, d2z, d3x, d3y, d3z;
            double a1 = (g[0] * x0 + g[1] * y0 + g[2] * z0) / mag0;
            if (a1 < 0) {
                d1x = g[0];
                d1y = g[1];
                d1z = g[2];
            }
            else {
                d1x = -g[0];
                d1y = -g[1];
                d1z = -g[2];
            }
            double a2 = (g[3] * x0 + g[4] * y0 + g[5] * z0) / mag0;
            if (a2 < 0) {
                d2x = g[3];
                d2y = g[4];
                d2z = g[5];
            }
            else {
                d2x = -g[3];
                d2y = -g[4];
                d2z = -g[5];
            }
            double a3 = (g[6] * x0 + g[7] * y0 + g[8] * z0) / mag0;
            if (a3 < 0) {
                d3x = g[6];
                d3y = g[7];
                d3z = g[8];
            }
            else {
                d3x = -g[6];
                d3y = -g[7];
                d3z = -g[8];
            }
            double u1x = d2x - d1x, u1y = d2y - d1y, u1z = d2z - d1z;
            double u2x = d3x - d1x, u2y = d3y - d1y, u2z = d3z - d1z;
            double uux = u1y * u2z - u1z * u2y;
            double uuy = u1z * u2x - u1x * u2z;
            double uuz = u1x * u2y - u1y * u2x;
            double ndem = sqrt(uux * uux + uuy * uuy + uuz * uuz);
            double nx = uux / ndem, ny = uuy / ndem, nz = uuz / ndem;
            double parat = (nx * x0 + ny * y0 + nz * z0) / (nx * d1x + ny * d1y + nz * d1z);
            float cdl = pow(pow(parat * d1x, 2.0) + pow(parat * d1y, 2.0) + pow(parat * d1z, 2.0), 0.5);
            table[26L * o + n] = cdl;
        }
    }
}

void build_growth_table(const Problem &p, int n_entries, std::vector<double> &growth) {
    // U after n updates is the n-fold float sum of du (src/CAupdate.cpp:236-237, U starts at 0);
    // the increment is min(0.045, max(0, A U^3 + B U^2 + C U + D)) with U capped at 210
    // (src/CAupdate.cpp:257-261), using this host's pow exactly as the reference does.
    growth.resize(n_entries);
    float u = 0.0f;
    for (int n = 0; n < n_entries; n++) {
        if (n > 0)
            u += p.du_value * (1);
        double LocU = u;
        LocU = std::min(210.0, LocU);
        double V = p.A_n * pow(LocU, 3.0) + p.B_n * pow(LocU, 2.0) + p.C_n * LocU + p.D_n;
        V = std::max(0.0, V);
        growth[n] = std::min(0.045, V);
    }
}

namespace {

inline long cell_index(const Geometry &g, int k, int i, int j) { return (long)k * g.mx * g.my + (long)i * g.my + j; }

// Single-rank decomposition: every strategy reduces to one rank owning nx x ny plus a ghost ring
// (src/CAfunctions.cpp:240-402 and 34-166 with np = 1).
void decompose(Problem &p, std::string &log) {
    InputConfig &c = p.cfg;
    Geometry &g = p.g;
    g.nx = c.nx;
    g.ny = c.ny;
    g.nz = c.nz;
    int strategy = c.decomposition_strategy;
    if (strategy == 2) {
        log += "Warning: Number of processors not divisible by two- defaulting to 1D decomposition\n";
        c.decomposition_strategy = 1;
    }
    else if (strategy == 3) {
        // sqrt(1) is a perfect square: 1 x 1 processors
        log += " Processors in X: 1 Processors in Y: 1\n";
    }
    g.procs_x = 1;
    g.procs_y = 1;
    g.mx = g.nx + 2;
    g.my = g.ny + 2;
    g.xoff = -1;
    g.yoff = -1;
    g.domain_size = (long)g.mx * g.my * g.nz;
}

// src/CAinitialize.cpp:1025-1055
void temp_init_directional(Problem &p) {
    Geometry &g = p.g;
    const InputConfig &c = p.cfg;
    g.zbound_low = 0;
    g.zbound_high = g.nz - 1;
    g.nz_active = g.nz;
    float du = c.R * c.deltat;
    for (int k = 0; k < g.nz; k++) {
        int cts = (int)(((k - 1) * c.G * c.deltax) / (c.R * c.deltat));
        for (int i = 0; i < g.mx; i++) {
            for (int j = 0; j < g.my; j++) {
                long idx = cell_index(g, k, i, j);
                p.layer_id[idx] = 0;
                p.du[idx] = du;
                p.cts[idx] = cts;
                int gx = i + g.xoff, gy = j + g.yoff;
                p.melted[idx] = (gx > -1 && gx < g.nx && gy > -1 && gy < g.ny && k > 0 && k < g.nz - 1) ? 1 : 0;
            }
        }
    }
}

// src/CAinitialize.cpp:1058-1124. Cells outside every spot keep CritTimeStep = 0 and
// UndercoolingChange = 0 (never written there; the reference's storage is fresh zero pages).
void temp_init_spots(Problem &p, std::string &log) {
    Geometry &g = p.g;
    const InputConfig &c = p.cfg;
    g.zbound_low = 0;
    g.zbound_high = c.spot_radius + 1;
    g.nz_active = c.spot_radius + 2;
    for (long idx = 0; idx < g.domain_size; idx++) {
        p.melted[idx] = 0;
        p.layer_id[idx] = -1;
        p.cts[idx] = 0;
        p.du[idx] = 0.0f;
    }
    int nspots = c.nspots_x * c.nspots_y;
    float iso_v = (c.R / c.G) * c.deltat / c.deltax;
    int time_between = c.spot_radius / iso_v + (c.freezing_range / c.R) / c.deltat;
    log += "Initializing temperature field for " + std::to_string(nspots) + " spots, each of which takes "
           "approximately " + std::to_string(time_between) + " time steps to solidify\n";
    float du = c.R * c.deltat;
    for (int layer = 0; layer < c.number_of_layers; layer++) {
        for (int n = 0; n < nspots; n++) {
            log += "Initializing spot " + std::to_string(n) + " on layer " + std::to_string(layer) + "\n";
            int xs = 2 + c.spot_radius + (n % c.nspots_x) * c.spot_offset;
            int ys = 2 + c.spot_radius + (n / c.nspots_x) * c.spot_offset;
            int zs = c.spot_radius + 2 + c.layer_height * layer;
            for (int k = 0; k < g.nz_active; k++) {
                float dz = (float)(zs - (k + c.layer_height * layer));
                for (int i = 0; i < g.mx; i++) {
                    float dxf = (float)(xs - (i + g.xoff));
                    for (int j = 0; j < g.my; j++) {
                        float dyf = (float)(ys - (j + g.yoff));
                        float dist = sqrtf(dxf * dxf + dyf * dyf + dz * dz);
                        if (dist <= c.spot_radius) {
                            long idx = (long)(k + layer * c.layer_height) * g.mx * g.my + (long)i * g.my + j;
                            p.cts[idx] = 1 + (int)(((float)(c.spot_radius) - dist) / iso_v) + time_between * n;
                            p.du[idx] = du;
                            p.layer_id[idx] = layer;
                            p.melted[idx] = 1;
                        }
                    }
                }
            }
        }
    }
}

// src/CAinitialize.cpp:1460-1529 (np = 1: rank seed 0, grain IDs 1, 2, ... in index order)
void substrate_constrained(Problem &p) {
    Geometry &g = p.g;
    std::mt19937_64 gen(0);
    std::uniform_real_distribution<double> dis(0.0, 1.0);
    for (int k = 0; k < g.nz; k++) {
        for (int i = 0; i < g.mx; i++) {
            for (int j = 0; j < g.my; j++) {
                int gx = i + g.xoff, gy = j + g.yoff;
                long idx = cell_index(g, k, i, j);
                if (gx == -1 || gx == g.nx || gy == -1 || gy == g.ny || k == 0 || k == g.nz - 1) {
                    p.cell_type[idx] = kWall;
                    p.grain_id[idx] = 0;
                }
                else if (k == 1 && i > 0 && i < g.mx - 1 && j > 0 && j < g.my - 1) {
                    double r = dis(gen);
                    p.cell_type[idx] = r < p.cfg.fract_surface_sites_active ? kActive : kLiquid;
                }
                else {
                    p.cell_type[idx] = kLiquid;
                }
            }
        }
    }
    int next_id = 1;
    for (long idx = 0; idx < g.domain_size; idx++)
        if (p.cell_type[idx] == kActive)
            p.grain_id[idx] = next_id++;
}

} // namespace

namespace {

// src/CAinitialize.cpp:1597-1732. The seeds are drawn here; the nearest-seed search for every
// substrate cell of the first layer runs on the device at admission (cells marked kVoronoiPending).
void substrate_from_spacing(Problem &p, std::vector<int32_t> &seeds, std::string &log) {
    Geometry &g = p.g;
    const InputConfig &c = p.cfg;
    std::mt19937_64 gen(1.0);
    std::uniform_real_distribution<double> dis(0.0, 1.0);
    float sp = c.substrate_grain_spacing;
    double prob = (c.deltax * c.deltax * c.deltax) / (sp * sp * sp * pow(10, -18));
    seeds.clear();
    for (int k = 1; k <= g.nz_active; k++)
        for (int i = 1; i < g.nx - 1; i++)
            for (int j = 1; j < g.ny - 1; j++) {
                double r = dis(gen);
                if (r < prob) {
                    seeds.push_back(i);
                    seeds.push_back(j);
                    seeds.push_back(k);
                }
            }
    int nseeds = (int)(seeds.size() / 3);
    log += "Number of baseplate grains: " + std::to_string(nseeds) + "\n";
    for (int k = 1; k < g.nz_active; k++)
        for (int i = 0; i < g.mx; i++)
            for (int j = 0; j < g.my; j++) {
                long idx = cell_index(g, k, i, j);
                p.grain_id[idx] = p.cts[idx] == 0 ? kVoronoiPending : 0;
            }
    log += "Baseplate grain structure initialized\n";
    for (int k = g.nz_active; k < g.nz; k++)
        for (int i = 1; i < g.mx - 1; i++)
            for (int j = 1; j < g.my - 1; j++) {
                long idx = cell_index(g, k, i, j);
                if (p.cts[idx] != 0)
                    p.grain_id[idx] = 0;
            }
    int next_id = nseeds + 1;
    for (long idx = (long)g.mx * g.my * g.nz_active; idx < g.domain_size; idx++)
        if (p.cts[idx] == 0)
            p.grain_id[idx] = next_id++;
    log += "Initialized baseplate and powder grain structure\n";
}

// src/CAinitialize.cpp:1736-1830
void active_cell_wall_init(Problem &p, const int it[9][26], const int lens[9], std::string &log) {
    Geometry &g = p.g;
    for (int k = 0; k < g.nz; k++)
        for (int i = 0; i < g.mx; i++)
            for (int j = 0; j < g.my; j++) {
                int gx = i + g.xoff, gy = j + g.yoff;
                long idx = cell_index(g, k, i, j);
                if (gx == -1 || gx == g.nx || gy == -1 || gy == g.ny || k == 0 || k == g.nz - 1) {
                    p.cell_type[idx] = kWall;
                    p.grain_id[idx] = 0;
                }
                if (p.cfg.extra_walls) {
                    if (gx == 0 || gx == g.nx - 1 || gy == 0 || gy == g.ny - 1 || gx == 1 || gx == g.nx - 2 ||
                        gy == 1 || gy == g.ny - 2) {
                        p.cell_type[idx] = kWall;
                        p.grain_id[idx] = 0;
                    }
                }
            }
    for (int k = 1; k < g.nz - 1; k++)
        for (int i = 0; i < g.mx; i++)
            for (int j = 0; j < g.my; j++) {
                long idx = cell_index(g, k, i, j);
                p.cell_type[idx] = p.cts[idx] == 0 ? kSolid : kLiquid;
            }
    long count = 0;
    for (int k = 1; k < g.nz - 1; k++)
        for (int j = 0; j < g.my; j++)
            for (int i = 0; i < g.mx; i++) {
                long idx = cell_index(g, k, i, j);
                if (p.cts[idx] != 0)
                    continue;
                int b = find_it_bounds(i, j, g.mx, g.my);
                for (int ll = 0; ll < lens[b]; ll++) {
                    int l = it[b][ll];
                    long nb = cell_index(g, k + kNeighborZ[l], i + kNeighborX[l], j + kNeighborY[l]);
                    if (p.cts[nb] > 0 && p.cell_type[nb] != kWall) {
                        p.cell_type[idx] = kActive;
                        p.du[idx] = p.du[nb];
                        count++;
                        break;
                    }
                }
            }
    log += "Number of substrate active cells across all ranks: " + std::to_string(count) + "\n";
}

// src/CAinitialize.cpp:1834-2206 (np = 1). The octahedron state of initially active cells is a
// per-cell function of (position, GrainID) and is filled in on the device at admission.
void grain_init(Problem &p, const int it[9][26], const int lens[9], std::string &log) {
    Geometry &g = p.g;
    std::mt19937_64 gen(0);
    std::uniform_real_distribution<double> dis(0.0, 1.0);
    double bulk_prob = p.cfg.nmax * p.cfg.deltax * p.cfg.deltax * p.cfg.deltax;
    int possible = 0;
    for (int k = 1; k < g.nz - 1; k++)
        for (int j = 1; j < g.my - 1; j++)
            for (int i = 1; i < g.mx - 1; i++) {
                long idx = cell_index(g, k, i, j);
                if (p.cts[idx] != 0) {
                    double r = dis(gen);
                    if (r < bulk_prob) {
                        possible++;
                        p.cell_type[idx] = kTemporaryInit;
                    }
                }
            }
    log += "Number of potential nucleated grains: " + std::to_string(possible) + "\n";
    int ncounter = -1;
    for (long idx = (long)g.mx * g.my; idx < (long)g.mx * g.my * (g.nz - 1); idx++)
        if (p.cell_type[idx] == kTemporaryInit)
            p.grain_id[idx] = ncounter--;
    // liquid cells with no non-solid, non-wall neighbour become solid, in the reference's order
    for (int k = 1; k < g.nz - 1; k++)
        for (int i = 1; i < g.mx - 1; i++)
            for (int j = 1; j < g.my - 1; j++) {
                long idx = cell_index(g, k, i, j);
                if (p.cell_type[idx] != kLiquid)
                    continue;
                int b = find_it_bounds(i, j, g.mx, g.my);
                bool any = false;
                for (int ll = 0; ll < lens[b] && !any; ll++) {
                    int l = it[b][ll];
                    int8_t t = p.cell_type[cell_index(g, k + kNeighborZ[l], i + kNeighborX[l], j + kNeighborY[l])];
                    any = (t != kSolid && t != kWall);
                }
                if (!any)
                    p.cell_type[idx] = kSolid;
            }
    p.possible_nuclei = possible;
}

// src/CAinitialize.cpp:2213-2247 and 2758-2768 (np = 1: no halo nuclei)
void nuclei_init(Problem &p, std::string &log) {
    Geometry &g = p.g;
    std::default_random_engine generator;
    std::normal_distribution<double> distribution(p.cfg.dTN, p.cfg.dTsigma);
    p.nuclei_loc.clear();
    p.nuclei_time.clear();
    for (long i = 0; i < g.domain_size; i++) {
        if (p.cell_type[i] == kTemporaryInit) {
            p.nuclei_loc.push_back((int32_t)i);
            double und = distribution(generator);
            int t = p.cts[i] + round(und / p.du[i]);
            p.nuclei_time.push_back(std::max(p.cts[i], t));
            p.cell_type[i] = kLiquid;
        }
    }
    log += "(0: " + std::to_string(p.nuclei_loc.size()) + ") ";
}

} // namespace

void initialize_problem(Problem &p, std::string &log) {
    auto t0 = std::chrono::steady_clock::now();
    InputConfig &c = p.cfg;
    if (c.simulation_type == "R")
        throw Unsupported("Problem type R (temperature data from files) is not supported by the B200 solver");
    if (c.simulation_type != "C" && c.simulation_type != "S")
        throw std::runtime_error("Unknown problem type \"" + c.simulation_type + "\"");
    if (c.number_of_layers < 1 || c.number_of_layers > 127)
        throw Unsupported("Number of layers must be between 1 and 127 (LayerID is stored in 8 bits)");
    if (c.simulation_type == "S" && c.use_substrate_file)
        throw Unsupported("Substrate files are not supported by the B200 solver");

    int it[9][26], lens[9];
    build_itlist(it, lens);
    decompose(p, log);
    Geometry &g = p.g;
    log += "Constrained solidification domain size: " + std::to_string(g.nx) + " by " + std::to_string(g.ny) +
           " by " + std::to_string(g.nz) + "\n";
    log += "================================================================\n";
    log += "Mesh initialized\n";
    if ((long)g.mx * g.my * g.nz > 2000000000L)
        throw Unsupported("domain too large: the cell index must fit in 31 bits");

    p.cts.assign(g.domain_size, 0);
    p.layer_id.assign(g.domain_size, 0);
    p.du.assign(g.domain_size, 0.0f);
    p.cell_type.assign(g.domain_size, 0);
    p.grain_id.assign(g.domain_size, 0);
    p.melted.assign(g.domain_size, 0);

    if (c.simulation_type == "C")
        temp_init_directional(p);
    else
        temp_init_spots(p, log);
    g.active_size = (long)g.mx * g.my * g.nz_active;
    log += "Done with temperature field initialization, active domain size is " + std::to_string(g.nz_active) +
           " out of " + std::to_string(g.nz) + " cells in the Z direction\n";

    read_orientations(c.orientation_file, p.guv);
    build_cdl_table(p.guv, p.cdl_table);
    log += "Done with orientation initialization \n";

    std::vector<int32_t> seeds;
    if (c.simulation_type == "C") {
        substrate_constrained(p);
    }
    else {
        substrate_from_spacing(p, seeds, log);
        active_cell_wall_init(p, it, lens, log);
    }
    grain_init(p, it, lens, log);
    log += "Grain struct initialized\n";
    log += " Possible nucleation events (rank: # events): \n";
    nuclei_init(p, log);
    log += "Nucleation initialized\n";

    // A, B, C normalised by dt/dx; D is left as read (src/runCA.cpp:198-200)
    p.A_n = c.A * c.deltat / c.deltax;
    p.B_n = c.B * c.deltat / c.deltax;
    p.C_n = c.C * c.deltat / c.deltax;
    p.D_n = c.D;

    // The device growth model needs every cell's UndercoolingChange to be 0 or one common value.
    float common = 0.0f;
    for (long i = 0; i < g.domain_size; i++) {
        float v = p.du[i];
        if (v == 0.0f)
            continue;
        if (common == 0.0f)
            common = v;
        else if (v != common)
            throw Unsupported("non-uniform UndercoolingChange is not supported by the B200 solver");
    }
    p.du_value = common;
    p.voronoi_seeds = seeds;
    p.init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace exaca
