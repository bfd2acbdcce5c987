// Host-side problem set-up for the B200 solver: geometry, temperature field, substrate, grain seeds,
// nuclei, and the lookup tables the device kernels use.
//
// The random streams are the reference's (libstdc++ mt19937_64 / uniform_real_distribution, drawn
// through the bit-identical Mt64 / uniform01 of rng.hpp; default_random_engine /
// normal_distribution) drawn in the reference's loop orders, so the same input file yields the same
// seeds and nuclei. Everything that is a pure per-cell function of these
// (the fresh-octahedron state of initially active cells, the Voronoi baseplate) is finished on the
// device when the problem is admitted to a pool.
#include "exaca_host.hpp"
#include "rng.hpp"

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <future>
#include <map>
#include <mutex>
#include <random>
#include <sstream>
#include <sys/stat.h>

namespace exaca {

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

namespace {

// The orientation file's unit vectors and fresh-octahedron critical lengths depend on the file
// alone, so they are read and tabulated once per process for each file (path, size and modification
// time) and shared by every problem that names it.
struct OrientationTables {
    std::vector<float> guv, cdl_table;
};

std::shared_ptr<const OrientationTables> orientation_tables(const std::string &path) {
    static std::mutex mu;
    static std::map<std::string, std::shared_ptr<const OrientationTables>> cache;
    struct stat st;
    std::string key = path;
    if (stat(path.c_str(), &st) == 0)
        key += "|" + std::to_string((long long)st.st_size) + "|" + std::to_string((long long)st.st_mtime);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end())
            return it->second;
    }
    auto t = std::make_shared<OrientationTables>();
    read_orientations(path, t->guv);
    build_cdl_table(t->guv, t->cdl_table);
    std::lock_guard<std::mutex> lock(mu);
    return cache.emplace(key, t).first->second;
}

} // namespace

void build_growth_table(const Problem &p, int n_entries, std::vector<double> &growth) {
    growth.resize(n_entries);
    build_growth_table(p, p.du_value, n_entries, growth.data());
}

void build_growth_table(const Problem &p, float du, int n_entries, double *growth) {
    // U after n updates is the n-fold float sum of du (src/CAupdate.cpp:236-237, U starts at 0);
    // the increment is min(0.045, max(0, A U^3 + B U^2 + C U + D)) with U capped at 210
    // (src/CAupdate.cpp:257-261), using this host's pow exactly as the reference does.
    float u = 0.0f;
    for (int n = 0; n < n_entries; n++) {
        if (n > 0)
            u += du * (1);
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

// ---- type R: reduced temperature data from files ------------------------------------------------

struct TemperatureData {
    std::vector<double> raw;        // the stored points, 6 values each: x, y, z, tm, tl, cr (RawData)
    std::vector<long> first, last;  // per layer: its range of raw
    std::vector<float> zmin_layer, zmax_layer;
    float xmin = 1000000.0f, ymin = 1000000.0f, zmin = 1000000.0f;
    float xmax = -1000000.0f, ymax = -1000000.0f, zmax = -1000000.0f;
};

// src/CAinitialize.cpp:135-146: the first n-1 comma-separated fields, then the rest of the line
void split_commas(std::string line, std::vector<std::string> &out) {
    for (size_t n = 0; n + 1 < out.size(); n++) {
        size_t pos = line.find(',');
        out[n] = line.substr(0, pos);
        line = line.substr(pos + 1, std::string::npos);
    }
    out.back() = line;
}

// src/CAinitialize.cpp:149-175: columns x, y, z, tm, tl (or ts), cr (or r), case-insensitive
void check_temperature_header(const std::string &line) {
    std::vector<std::string> v(6);
    split_commas(line, v);
    static const std::vector<std::vector<std::string>> expected = {{"x"}, {"y"}, {"z"}, {"tm"}, {"tl", "ts"}, {"r", "cr"}};
    for (size_t n = 0; n < 6; n++) {
        std::string val;
        for (char ch : v[n])
            if (!std::isspace((unsigned char)ch))
                val += (char)std::tolower((unsigned char)ch);
        if (std::find(expected[n].begin(), expected[n].end(), val) == expected[n].end())
            throw std::runtime_error(expected[n].back() + " not found in temperature file header");
    }
}

// src/CAinitialize.cpp:177-187: the first pt.size() values of a data line, as std::stod reads them
void temperature_point(const std::string &line, std::vector<double> &pt) {
    std::vector<std::string> v(pt.size());
    split_commas(line, v);
    for (size_t n = 0; n < pt.size(); n++)
        pt[n] = std::stod(v[n]);
}

std::string dstr(double v) {
    std::ostringstream s;
    s << v;
    return s.str();
}

// x/y range of the temperature grid one rank reads (src/CAinitialize.cpp:906-923, 1171-1188)
void read_bounds(const Geometry &g, int ratio, int &lx, int &ly, int &ux, int &uy) {
    lx = g.xoff <= 2 ? 2 : g.xoff - ((g.xoff - 2) % ratio);
    ly = g.yoff <= 2 ? 2 : g.yoff - ((g.yoff - 2) % ratio);
    ux = (g.xoff + g.mx - 1 >= g.nx - 3) ? g.nx - 3 : g.xoff + g.mx - 1 + ratio - ((g.xoff + (g.mx - 1) - 2) % ratio);
    uy = (g.yoff + g.my - 1 >= g.ny - 3) ? g.ny - 3 : g.yoff + g.my - 1 + ratio - ((g.yoff + (g.my - 1) - 2) % ratio);
}

// ParallelMeshInit for type R (src/CAinitialize.cpp:747-1003): the domain bounds from every file's
// points, the decomposition, then the points of this rank's x/y range.
void mesh_init_reduced(Problem &p, TemperatureData &td, std::string &log) {
    InputConfig &c = p.cfg;
    const int nfiles = c.temp_files_in_series, layers = c.number_of_layers;
    std::vector<std::string> paths(nfiles);
    for (int i = 1; i <= nfiles; i++)
        paths[i - 1] = c.temppath + "/" + (nfiles > 1 ? std::to_string(i) + c.tempfile : c.tempfile);
    const int ratio_read = c.ht_deltax / c.deltax; // truncation, as the reference
    {
        std::ifstream f(paths[0]);
        std::string line;
        std::getline(f, line);
        if (line.find("Number of temperature data points") != std::string::npos)
            throw std::runtime_error("Error: Old header and temperature file format no longer supported");
    }
    const int to_read = std::min(layers, nfiles);
    td.zmin_layer.assign(layers, 0.0f);
    td.zmax_layer.assign(layers, 0.0f);
    td.first.assign(layers, 0);
    td.last.assign(layers, 0);
    for (int L = 1; L <= to_read; L++) {
        std::ifstream f(paths[L - 1]);
        std::string header;
        std::getline(f, header);
        check_temperature_header(header);
        std::vector<double> X, Y, Z, pt(3);
        while (!f.eof()) {
            std::string line;
            std::getline(f, line);
            if (line.empty())
                break;
            temperature_point(line, pt);
            X.push_back(pt[0]);
            Y.push_back(pt[1]);
            Z.push_back(pt[2]);
        }
        if (X.empty())
            throw std::runtime_error("Temperature file " + paths[L - 1] + " holds no data points");
        double x0 = *std::min_element(X.begin(), X.end()), x1 = *std::max_element(X.begin(), X.end());
        double y0 = *std::min_element(Y.begin(), Y.end()), y1 = *std::max_element(Y.begin(), Y.end());
        double z0 = *std::min_element(Z.begin(), Z.end()), z1 = *std::max_element(Z.begin(), Z.end());
        z0 += c.deltax * c.layer_height * (L - 1);
        z1 += c.deltax * c.layer_height * (L - 1);
        if (x0 < td.xmin)
            td.xmin = x0;
        if (x1 > td.xmax)
            td.xmax = x1;
        if (y0 < td.ymin)
            td.ymin = y0;
        if (y1 > td.ymax)
            td.ymax = y1;
        if (z0 < td.zmin)
            td.zmin = z0;
        if (z1 > td.zmax)
            td.zmax = z1;
        td.zmin_layer[L - 1] = z0;
        td.zmax_layer[L - 1] = z1;
        log += "Layer = " + std::to_string(L) + " Z Bounds are " + dstr(z0) + " " + dstr(z1) + "\n";
    }
    // layers beyond the files repeat them, shifted up by the layer offset
    for (int L = nfiles; L < layers; L++) {
        if (nfiles == 1) {
            td.zmin_layer[L] = td.zmin_layer[L - 1] + c.deltax * c.layer_height;
            td.zmax_layer[L] = td.zmax_layer[L - 1] + c.deltax * c.layer_height;
        }
        else {
            const int rep = L % nfiles, unit = L / nfiles;
            td.zmin_layer[L] = td.zmin_layer[rep] + unit * nfiles * c.deltax * c.layer_height;
            td.zmax_layer[L] = td.zmax_layer[rep] + unit * nfiles * c.deltax * c.layer_height;
        }
        td.zmax += c.deltax * c.layer_height;
    }
    // wall + solid ring at each x/y side, wall + one row at the bottom, wall at the top
    c.nx = round((td.xmax - td.xmin) / c.deltax) + 1 + 4;
    c.ny = round((td.ymax - td.ymin) / c.deltax) + 1 + 4;
    c.nz = round((td.zmax - td.zmin) / c.deltax) + 1 + 3;
    log += "Domain size: " + std::to_string(c.nx) + " by " + std::to_string(c.ny) + " by " + std::to_string(c.nz) + "\n";
    log += "X Limits of domain: " + dstr(td.xmin) + " and " + dstr(td.xmax) + "\n";
    log += "Y Limits of domain: " + dstr(td.ymin) + " and " + dstr(td.ymax) + "\n";
    log += "Z Limits of domain: " + dstr(td.zmin) + " and " + dstr(td.zmax) + "\n";
    log += "================================================================\n";
    decompose(p, log);
    int lx, ly, ux, uy;
    read_bounds(p.g, ratio_read, lx, ly, ux, uy);
    for (int L = 1; L <= to_read; L++) {
        std::ifstream f(paths[L - 1]);
        td.first[L - 1] = (long)td.raw.size();
        std::string line;
        std::getline(f, line); // header
        std::vector<double> pt(6);
        while (!f.eof()) {
            std::getline(f, line);
            if (line.empty())
                break;
            temperature_point(line, pt);
            const int xi = round((pt[0] - td.xmin) / c.deltax) + 2;
            const int yi = round((pt[1] - td.ymin) / c.deltax) + 2;
            if (xi >= lx && xi <= ux && yi >= ly && yi <= uy)
                td.raw.insert(td.raw.end(), pt.begin(), pt.end());
        }
        td.last[L - 1] = (long)td.raw.size();
    }
    for (int L = nfiles; L < layers; L++) {
        const int from = nfiles == 1 ? L - 1 : L % nfiles;
        td.first[L] = td.first[from];
        td.last[L] = td.last[from];
    }
}

// TempInit_Reduced (src/CAinitialize.cpp:1128-1405): per layer, the last liquidus time and the
// cooling rate of every temperature point, trilinear interpolation onto the CA grid when the
// temperature grid is coarser, then CritTimeStep, UndercoolingChange, LayerID and Melted of the
// cells whose normalised liquidus time is positive, and the layer's finish time step.
void temp_init_reduced(Problem &p, const TemperatureData &td, std::string &log) {
    InputConfig &c = p.cfg;
    Geometry &g = p.g;
    const double unrounded = c.ht_deltax / c.deltax, fl = floor(unrounded);
    if (unrounded - fl > 0.0005)
        throw std::runtime_error("Error: Temperature data point spacing not evenly divisible by CA cell size");
    else if (unrounded - fl > 0.000001)
        log += "Note: Adjusting cell size from " + dstr(c.deltax) + " to " + dstr(c.ht_deltax / fl) +
               " to ensure even divisibility of CA cell size into temperature data spacing\n";
    c.deltax = c.ht_deltax / fl;
    const int ratio = round(c.ht_deltax / c.deltax);
    int lx, ly, ux, uy;
    read_bounds(g, ratio, lx, ly, ux, uy);
    for (long i = 0; i < g.domain_size; i++) {
        p.melted[i] = 0;
        p.layer_id[i] = -1;
    }
    const int layers = c.number_of_layers;
    p.finish_time_step.assign(layers, 0);
    const int sx = ux - lx + 1, sy = uy - ly + 1;
    for (int L = 0; L < layers; L++) {
        double smallest = 1000000000, largest = 0;
        const int nzt = round((td.zmax_layer[L] - td.zmin_layer[L]) / c.deltax) + 1;
        log += "Initializing temporary temperature data structures with " + std::to_string(nzt) +
               " cells in z direction\n";
        log += "Layer " + std::to_string(L) + " rank 0 ZMin this layer is " + dstr(td.zmin_layer[L]) + "\n";
        std::vector<double> CR((size_t)nzt * sx * sy, -1.0), TL((size_t)nzt * sx * sy, -1.0);
        auto at = [&](int z, int x, int y) -> size_t {
            if (z < 0 || z >= nzt || x < 0 || x >= sx || y < 0 || y >= sy)
                throw std::runtime_error("temperature data point outside the layer's temperature grid");
            return ((size_t)z * sx + x) * sy + y;
        };
        const long start = td.first[L], end = td.last[L];
        log += "Range for layer " + std::to_string(L) + " on rank 0 is " + std::to_string(start) + " to " +
               std::to_string(end) + "\n";
        int xi = -1, yi = -1, zi = -1;
        for (long i = start; i < end; i++) {
            const int pos = (int)(i % 6);
            if (pos == 0) {
                xi = round((td.raw[i] - td.xmin) / c.deltax) + 2;
            }
            else if (pos == 1) {
                yi = round((td.raw[i] - td.ymin) / c.deltax) + 2;
            }
            else if (pos == 2) {
                zi = round((td.raw[i] + c.deltax * c.layer_height * L - td.zmin_layer[L]) / c.deltax);
            }
            else if (pos == 4) {
                // only the last time the point goes below the liquidus counts
                const size_t q = at(zi, xi - lx, yi - ly);
                if (td.raw[i] > TL[q]) {
                    TL[q] = td.raw[i];
                    if (td.raw[i] < smallest)
                        smallest = td.raw[i];
                }
                else {
                    i = i + 1; // skip this point's cooling rate
                }
            }
            else if (pos == 5) {
                const size_t q = at(zi, xi - lx, yi - ly);
                CR[q] = td.raw[i];
                float solidus = TL[q] + c.freezing_range / CR[q];
                if (solidus > largest)
                    largest = solidus;
            }
        }
        log += "Smallest time globally for layer " + std::to_string(L) + " is " + dstr(smallest) + "\n";
        log += "Largest time globally for layer " + std::to_string(L) + " is " + dstr(largest) + "\n";
        p.finish_time_step[L] = round((largest - smallest) / c.deltat);
        log += " Layer " + std::to_string(L) + " FINISH TIME STEP IS " + std::to_string(p.finish_time_step[L]) + "\n";
        log += "Layer " + std::to_string(L) + " temperatures read\n";
        if (ratio != 1) {
            // in place, in the reference's loop order (later cells may read interpolated values)
            for (int k = 0; k < nzt; k++) {
                const int lowz = k - (k % ratio);
                int highz = lowz + ratio;
                const double fhz = (double)(k - lowz) / (double)(ratio), flz = 1.0 - fhz;
                if (highz > nzt - 1)
                    highz = lowz;
                for (int i = 0; i <= ux - lx; i++) {
                    const int lowx = i - (i % ratio);
                    int highx = lowx + ratio;
                    const double fhx = (double)(i - lowx) / (double)(ratio), flx = 1.0 - fhx;
                    if (highx >= ux - lx)
                        highx = ux - lx;
                    for (int j = 0; j <= uy - ly; j++) {
                        const int lowy = j - (j % ratio);
                        int highy = lowy + ratio;
                        const double fhy = (float)(j - lowy) / (float)(ratio), fly = 1.0 - fhy;
                        if (highy >= uy - ly)
                            highy = uy - ly;
                        for (std::vector<double> *F : {&TL, &CR}) {
                            std::vector<double> &A = *F;
                            const double p1 = A[at(lowz, lowx, lowy)], p2 = A[at(lowz, highx, lowy)];
                            const double p12 = flx * p1 + fhx * p2;
                            const double p3 = A[at(lowz, lowx, highy)], p4 = A[at(lowz, highx, highy)];
                            const double p34 = flx * p3 + fhx * p4;
                            const double p1234 = p12 * fly + p34 * fhy;
                            const double p5 = A[at(highz, lowx, lowy)], p6 = A[at(highz, highx, lowy)];
                            const double p56 = flx * p5 + fhx * p6;
                            const double p7 = A[at(highz, lowx, highy)], p8 = A[at(highz, highx, highy)];
                            const double p78 = flx * p7 + fhx * p8;
                            const double p5678 = p56 * fly + p78 * fhy;
                            if (p1 > 0 && p2 > 0 && p3 > 0 && p4 > 0 && p5 > 0 && p6 > 0 && p7 > 0 && p8 > 0)
                                A[at(k, i, j)] = p1234 * flz + p5678 * fhz;
                        }
                    }
                }
            }
        }
        log += "Interpolation done\n";
        const int zbase = round((td.zmin_layer[L] - td.zmin) / c.deltax) + 2;
        if (L == 0) {
            g.zbound_low = 0;
            g.zbound_high = zbase + nzt - 1;
            g.nz_active = g.zbound_high - g.zbound_low + 1;
        }
        log += "Layer " + std::to_string(L) + " data belongs to global z coordinates of " + std::to_string(zbase) +
               " through " + std::to_string(zbase + nzt - 1) + "\n";
        for (int k = 0; k < nzt; k++)
            for (int ii = lx; ii <= ux; ii++)
                for (int jj = ly; jj <= uy; jj++) {
                    if (ii < g.xoff || ii >= g.xoff + g.mx || jj < g.yoff || jj >= g.yoff + g.my)
                        continue;
                    const size_t q = at(k, ii - lx, jj - ly);
                    // liquidus time from the start of the layer
                    const double ctl = TL[q] - smallest;
                    if (ctl > 0) {
                        const int z = zbase + k;
                        if (z < 0 || z >= g.nz)
                            throw std::runtime_error("temperature data outside the domain in z");
                        const long idx = (long)z * g.mx * g.my + (long)(ii - g.xoff) * g.my + (jj - g.yoff);
                        p.melted[idx] = 1;
                        p.cts[idx] = round(ctl / c.deltat);
                        p.layer_id[idx] = L;
                        p.du[idx] = std::abs(CR[q]) * c.deltat;
                    }
                }
    }
    log += "First layer Z bounds are " + std::to_string(g.zbound_low) + " and " + std::to_string(g.zbound_high) + "\n";
}

// src/CAinitialize.cpp:1460-1529 (np = 1: rank seed 0, grain IDs 1, 2, ... in index order)
void substrate_constrained(Problem &p) {
    Geometry &g = p.g;
    Mt64 gen(0);
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
                    double r = uniform01(gen.next());
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
    Mt64 gen((uint64_t)1.0); // std::mt19937_64 gen(1.0)
    float sp = c.substrate_grain_spacing;
    double prob = (c.deltax * c.deltax * c.deltax) / (sp * sp * sp * pow(10, -18));
    seeds.clear();
    for (int k = 1; k <= g.nz_active; k++)
        for (int i = 1; i < g.nx - 1; i++)
            for (int j = 1; j < g.ny - 1; j++) {
                double r = uniform01(gen.next());
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
    Mt64 gen(0);
    double bulk_prob = p.cfg.nmax * p.cfg.deltax * p.cfg.deltax * p.cfg.deltax;
    int possible = 0;
    for (int k = 1; k < g.nz - 1; k++)
        for (int j = 1; j < g.my - 1; j++)
            for (int i = 1; i < g.mx - 1; i++) {
                long idx = cell_index(g, k, i, j);
                if (p.cts[idx] != 0) {
                    double r = uniform01(gen.next());
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

// Type C without the per-cell host fields (src/CAinitialize.cpp:1025-1055, 1460-1529, 1834-2247):
// the plane CritTimeSteps, the substrate seeds and the nuclei come from the same random streams
// in the same orders as the dense path above; the dense fields are made from them on the device at
// admission (and by materialize_fields on the host).
void init_directional_seeds(Problem &p, std::string & /* log: type C adds no notes */) {
    Geometry &g = p.g;
    const InputConfig &c = p.cfg;
    g.zbound_low = 0;
    g.zbound_high = g.nz - 1;
    g.nz_active = g.nz;
    DirectionalSeeds &d = p.dir;
    d.used = true;
    d.plane_cts.resize(g.nz);
    for (int k = 0; k < g.nz; k++)
        d.plane_cts[k] = (int)(((k - 1) * c.G * c.deltax) / (c.R * c.deltat));
    p.du_value = c.R * c.deltat;
    // substrate: one draw per cell of plane k = 1 inside the ghost ring, in (i, j) order
    {
        Mt64 gen(0);
        d.active.clear();
        for (int i = 1; i < g.mx - 1; i++)
            for (int j = 1; j < g.my - 1; j++)
                if (uniform01(gen.next()) < c.fract_surface_sites_active)
                    d.active.push_back(cell_index(g, 1, i, j));
    }
    // potential nuclei: one draw per cell with CritTimeStep != 0, planes k = 1 .. nz-2 in (k, j, i)
    // order; numbered -1, -2, ... in index order
    std::vector<int32_t> sites;
    {
        Mt64 gen(0);
        const double bulk_prob = c.nmax * c.deltax * c.deltax * c.deltax;
        const int ni = g.mx - 2, nj = g.my - 2;
        const bool by_limit = bulk_prob > 0.0 && bulk_prob <= 0.5;
        const uint64_t x_lim = by_limit ? uniform01_limit(bulk_prob) : 0;
        for (int k = 1; k < g.nz - 1; k++) {
            if (d.plane_cts[k] == 0)
                continue;
            if (by_limit) {
                // the plane's draws in (j, i) order, scanned for outputs below the probability's limit
                gen.scan_below((uint64_t)ni * nj, x_lim, [&](uint64_t t) {
                    const int j = 1 + (int)(t / ni), i = 1 + (int)(t % ni);
                    sites.push_back((int32_t)cell_index(g, k, i, j));
                });
            }
            else {
                for (int j = 1; j < g.my - 1; j++)
                    for (int i = 1; i < g.mx - 1; i++)
                        if (uniform01(gen.next()) < bulk_prob)
                            sites.push_back((int32_t)cell_index(g, k, i, j));
            }
        }
    }
    std::sort(sites.begin(), sites.end());
    {
        std::default_random_engine generator;
        std::normal_distribution<double> distribution(c.dTN, c.dTsigma);
        p.nuclei_loc = sites;
        p.nuclei_time.resize(sites.size());
        for (size_t n = 0; n < sites.size(); n++) {
            const int cts = d.plane_cts[sites[n] / (g.mx * g.my)];
            const double und = distribution(generator);
            const int t = cts + round(und / p.du_value);
            p.nuclei_time[n] = std::max(cts, t);
        }
    }
    p.possible_nuclei = (int)sites.size();
}

} // namespace

void materialize_fields(const Problem &p) {
    if (!p.dir.used)
        return;
    std::lock_guard<std::mutex> lock(*p.fields_mutex);
    if (!p.cell_type.empty())
        return;
    const Geometry &g = p.g;
    const long N = g.domain_size;
    p.cts.resize(N);
    p.layer_id.assign(N, 0);
    p.du.assign(N, p.du_value);
    p.cell_type.resize(N);
    p.grain_id.assign(N, 0);
    p.melted.resize(N);
    for (int k = 0; k < g.nz; k++)
        for (int i = 0; i < g.mx; i++)
            for (int j = 0; j < g.my; j++) {
                const long idx = cell_index(g, k, i, j);
                const bool wall = i == 0 || i == g.mx - 1 || j == 0 || j == g.my - 1 || k == 0 || k == g.nz - 1;
                p.cts[idx] = p.dir.plane_cts[k];
                p.cell_type[idx] = wall ? kWall : kLiquid;
                p.melted[idx] = wall ? 0 : 1;
            }
    for (size_t n = 0; n < p.dir.active.size(); n++) {
        p.cell_type[p.dir.active[n]] = kActive;
        p.grain_id[p.dir.active[n]] = (int32_t)(n + 1);
    }
    for (size_t n = 0; n < p.nuclei_loc.size(); n++)
        p.grain_id[p.nuclei_loc[n]] = -(int32_t)(n + 1);
}

void initialize_problem(Problem &p, std::string &log) {
    auto t0 = std::chrono::steady_clock::now();
    InputConfig &c = p.cfg;
    const bool type_r = c.simulation_type == "R";
    if (c.simulation_type != "C" && c.simulation_type != "S" && !type_r)
        throw std::runtime_error("Unknown problem type \"" + c.simulation_type + "\"");
    if (c.number_of_layers < 1 || c.number_of_layers > 127)
        throw Unsupported("Number of layers must be between 1 and 127 (LayerID is stored in 8 bits)");
    if (c.simulation_type != "C" && c.use_substrate_file)
        throw Unsupported("Substrate files are not supported by the B200 solver");

    int it[9][26], lens[9];
    build_itlist(it, lens);
    TemperatureData td;
    if (type_r) {
        mesh_init_reduced(p, td, log);
    }
    else {
        decompose(p, log);
        log += "Constrained solidification domain size: " + std::to_string(p.g.nx) + " by " +
               std::to_string(p.g.ny) + " by " + std::to_string(p.g.nz) + "\n";
        log += "================================================================\n";
    }
    Geometry &g = p.g;
    log += "Mesh initialized\n";
    if ((long)g.mx * g.my * g.nz > 2000000000L)
        throw Unsupported("domain too large: the cell index must fit in 31 bits");

    // Type C with more than one interior cell (then no liquid cell is cut off by walls) keeps no
    // per-cell host fields: they are made on the device
    const bool seeds_only = c.simulation_type == "C" && (g.nx > 3 || g.ny > 3 || g.nz > 3);
    if (seeds_only) {
        // the orientation tables are read (or taken from the process's cache) while the seeds are drawn
        auto tables = std::async(std::launch::async, orientation_tables, c.orientation_file);
        init_directional_seeds(p, log);
        g.active_size = (long)g.mx * g.my * g.nz_active;
        log += "Done with temperature field initialization, active domain size is " + std::to_string(g.nz_active) +
               " out of " + std::to_string(g.nz) + " cells in the Z direction\n";
        {
            auto t = tables.get();
            p.guv = t->guv;
            p.cdl_table = t->cdl_table;
        }
        log += "Done with orientation initialization \n";
        log += "Number of potential nucleated grains: " + std::to_string(p.nuclei_loc.size()) + "\n";
        log += "Grain struct initialized\n";
        log += " Possible nucleation events (rank: # events): \n";
        log += "(0: " + std::to_string(p.nuclei_loc.size()) + ") ";
        log += "Nucleation initialized\n";
        p.A_n = c.A * c.deltat / c.deltax;
        p.B_n = c.B * c.deltat / c.deltax;
        p.C_n = c.C * c.deltat / c.deltax;
        p.D_n = c.D;
        p.du_values.clear();
        p.du_class.clear();
        p.init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return;
    }
    p.cts.assign(g.domain_size, 0);
    p.layer_id.assign(g.domain_size, 0);
    p.du.assign(g.domain_size, 0.0f);
    p.cell_type.assign(g.domain_size, 0);
    p.grain_id.assign(g.domain_size, 0);
    p.melted.assign(g.domain_size, 0);

    if (c.simulation_type == "C")
        temp_init_directional(p);
    else if (type_r)
        temp_init_reduced(p, td, log);
    else
        temp_init_spots(p, log);
    td = TemperatureData(); // the raw temperature points are not needed past this point
    g.active_size = (long)g.mx * g.my * g.nz_active;
    log += "Done with temperature field initialization, active domain size is " + std::to_string(g.nz_active) +
           " out of " + std::to_string(g.nz) + " cells in the Z direction\n";

    {
        auto t = orientation_tables(c.orientation_file);
        p.guv = t->guv;
        p.cdl_table = t->cdl_table;
    }
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

    // The device growth model reads one growth table per distinct non-zero UndercoolingChange value
    // (types C and S have one; type R one per cooling rate after interpolation).
    std::vector<float> values;
    for (long i = 0; i < g.domain_size; i++)
        if (p.du[i] != 0.0f)
            values.push_back(p.du[i]);
    std::sort(values.begin(), values.end());
    values.erase(std::unique(values.begin(), values.end()), values.end());
    if ((int)values.size() > kMaxUndercoolingValues)
        throw Unsupported("the temperature data give " + std::to_string(values.size()) +
                          " distinct UndercoolingChange values; the B200 solver holds at most " +
                          std::to_string(kMaxUndercoolingValues) + " growth tables");
    p.du_value = values.empty() ? 0.0f : values[0];
    p.du_values.clear();
    p.du_class.clear();
    if (values.size() > 1) {
        p.du_values = values;
        p.du_class.assign(g.domain_size, 0);
        for (long i = 0; i < g.domain_size; i++)
            if (p.du[i] != 0.0f)
                p.du_class[i] = (uint16_t)(std::lower_bound(values.begin(), values.end(), p.du[i]) - values.begin());
    }
    p.voronoi_seeds = seeds;
    p.init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace exaca
