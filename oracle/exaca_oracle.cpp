// Test infrastructure only: a serial CPU restatement of the ExaCA reference's per-cycle update and
// of the initialisation it needs, used by the tests as the checker of the CUDA solver. It is never
// linked into or called by the product.
//
// Parity: pinned. tests/test_oracle.py checks this restatement bit for bit against the final
// GrainID / CellType arrays, final cycle and post-init fields of the reference itself (compiled
// from its unmodified sources against single-rank shims), stored in tests/golden/*.npz.
//
// Problem types C, S and R (temperature files), one or several layers; no substrate files.
//
// The restatement follows the reference's loops literally, in its serial (Kokkos-Serial) order:
// every function cites the reference lines it follows (paths relative to the reference project).
// The arithmetic is the reference's: same types, same operation order, libm pow/sqrt/sqrtf, the
// libstdc++ random engines and distributions; compiled with -ffp-contract=off.
//
// C ABI (for ctypes):
//   void *oracle_create(const char *input_file, const char *data_dir)   NULL on error
//   const char *oracle_error(void)
//   int  oracle_geometry(void *o, long long *out6)    mx, my, nz, nz_active, domain size, active size
//                                                      (of the current layer's window)
//   int  oracle_step(void *o, int n_cycles)            n raw cycles of the current layer (no check)
//   int  oracle_run_to(void *o, int stop, int *final)   the same, paused (returns 1) after cycle `stop`
//   int  oracle_run(void *o, int *final_cycle)          to termination of the last layer, as
//                                                      RunProgram_Reduced does
//   int  oracle_cycle(void *o)
//   void oracle_set_threads(int n)                     host threads of CellCapture's first pass
//   int  oracle_census(void *o, long long *out, int max)  censuses of oracle_run (6 numbers each)
//   int  oracle_fields(void *o, int *cell_type, int *grain_id, float *dl, float *doc, float *cdl)
//   void oracle_free(void *o)
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

enum { Wall = 0, Solid = 1, Active = 2, TemporaryUpdate = 3, TemporaryInit = 4, Liquid = 5 };
const int NGrainOrientations = 10000;

thread_local std::string g_error;
// host threads of the dense first pass of CellCapture (oracle_set_threads; 1 = plain serial loop)
int g_threads = 1;

// ---- input file (src/CAinitialize.cpp:24-576) ---------------------------------------------------
struct Input {
    std::string type;
    double A, B, C, D, freezing;
    double deltax, NMax, dTN, dTsigma, deltat, G, R, fract;
    int nx, ny, nz, nspx, nspy, spot_offset, spot_radius, layers, layer_height;
    float grain_spacing;
    std::string orientation_file;
    // type R
    double ht_deltax = 0;
    std::vector<std::string> temp_paths;
    bool extra_walls = false;
};

struct Reader {
    std::ifstream in;
    explicit Reader(const std::string &p) : in(p) {
        if (!in.is_open())
            throw std::runtime_error("cannot open " + p);
        std::string l;
        while (std::getline(in, l))
            if (l == "*****")
                break;
    }
    std::string last_key; // the key of the last value read
    // key check by substring (key, or alt when given); the value is everything after the colon,
    // whitespace removed
    std::string value(const std::string &key, const std::string &alt = "") {
        std::string line;
        for (;;) {
            if (!std::getline(in, line))
                throw std::runtime_error("missing key " + key);
            std::size_t c = line.find(':');
            if (c == std::string::npos)
                throw std::runtime_error("no colon in line: " + line);
            std::string k = line.substr(0, c);
            bool deprecated = k.find("Burst buffer") != std::string::npos &&
                              k.find("Source of input length unit") != std::string::npos;
            if (deprecated)
                continue;
            if (k.find(key) == std::string::npos && (alt.empty() || k.find(alt) == std::string::npos))
                throw std::runtime_error("expected key " + key);
            last_key = k;
            std::string v;
            for (char ch : line.substr(c + 1))
                if (!std::isspace((unsigned char)ch))
                    v.push_back(ch);
            return v;
        }
    }
};

Input read_input(const std::string &path, const std::string &data_dir) {
    Input I;
    Reader r(path);
    I.type = r.value("Problem type");
    r.value("Decomposition strategy");
    std::string material = r.value("Material");
    {
        Reader m(data_dir + "/Materials/" + material);
        I.A = atof(m.value("A").c_str());
        I.B = atof(m.value("B").c_str());
        I.C = atof(m.value("C").c_str());
        I.D = atof(m.value("D").c_str());
        I.freezing = atof(m.value("Alloy freezing range").c_str());
    }
    I.deltax = atof(r.value("Cell size").c_str()) * pow(10, -6);
    I.NMax = atof(r.value("Heterogeneous nucleation density").c_str()) * pow(10, 12);
    I.dTN = atof(r.value("Mean nucleation undercooling").c_str());
    I.dTsigma = atof(r.value("Standard deviation of nucleation undercooling").c_str());
    r.value("Path to output");
    r.value("Output file base name");
    I.orientation_file = data_dir + "/Substrate/" + r.value("File of grain orientations");
    I.layers = 1;
    if (I.type == "C") {
        I.G = atof(r.value("Thermal gradient").c_str());
        I.R = atof(r.value("Cooling rate").c_str());
        I.nx = std::stoi(r.value("Domain size in x")) + 2;
        I.ny = std::stoi(r.value("Domain size in y")) + 2;
        I.nz = std::stoi(r.value("Domain size in z")) + 2;
        int N = std::stoi(r.value("\"N\""));
        I.deltat = I.deltax / (N * (I.R / I.G));
        I.fract = atof(r.value("Fraction of surface sites active").c_str());
    }
    else if (I.type == "S") {
        I.G = atof(r.value("Thermal gradient").c_str());
        I.R = atof(r.value("Cooling rate").c_str());
        I.nspx = std::stoi(r.value("Number of spots in x"));
        I.nspy = std::stoi(r.value("Number of spots in y"));
        float off = atof(r.value("Offset between spot centers").c_str());
        I.spot_offset = off * 1.0 * pow(10, -6) / I.deltax;
        float rad = atof(r.value("Radii of spots").c_str());
        I.spot_radius = rad * 1.0 * pow(10, -6) / I.deltax;
        I.layers = std::stoi(r.value("Number of layers"));
        I.layer_height = std::stoi(r.value("Offset between layers"));
        int N = std::stoi(r.value("\"N\""));
        I.deltat = I.deltax / (N * (I.R / I.G));
        I.grain_spacing = atof(r.value("Substrate grain spacing").c_str());
        I.nz = I.spot_radius + 3 + (I.layers - 1) * I.layer_height;
        I.nx = 4 + 2 * I.spot_radius + I.spot_offset * (I.nspx - 1);
        I.ny = 4 + 2 * I.spot_radius + I.spot_offset * (I.nspy - 1);
    }
    else if (I.type == "R") {
        // src/CAinitialize.cpp:321-392
        I.ht_deltax = atof(r.value("Heat transport data mesh size").c_str()) * pow(10, -6);
        I.deltat = atof(r.value("Time step").c_str()) * pow(10, -6);
        std::string v = r.value("Path to substrate file", "Substrate grain spacing");
        if (r.last_key.find("Substrate grain spacing") == std::string::npos)
            throw std::runtime_error("oracle: substrate files are not restated");
        I.grain_spacing = atof(v.c_str());
        std::string path = r.value("Path to temperature file"), name = r.value("Temperature filename");
        int nfiles = std::stoi(r.value("Number of temperature files"));
        for (int i = 1; i <= nfiles; i++)
            I.temp_paths.push_back(path + "/" + (nfiles > 1 ? std::to_string(i) + name : name));
        I.extra_walls = r.value("Extra set of wall cells") == "Y";
        I.layers = std::stoi(r.value("Number of layers"));
        I.layer_height = std::stoi(r.value("Offset between layers"));
    }
    else {
        throw std::runtime_error("oracle: problem types C, S and R only");
    }
    return I;
}

// ---- type R temperature data (src/CAinitialize.cpp:135-198, 747-1003, 1128-1405) ------------------
// split at commas: the first n-1 fields, then the rest of the line (src/CAinitialize.cpp:135-146)
std::vector<double> temperature_values(std::string line, int n) {
    std::vector<double> out(n);
    for (int q = 0; q < n - 1; q++) {
        std::size_t pos = line.find(',');
        out[q] = std::stod(line.substr(0, pos));
        line = line.substr(pos + 1);
    }
    out[n - 1] = std::stod(line);
    return out;
}

struct TemperatureGrid {
    std::vector<double> raw; // 6 values per stored point (RawData)
    std::vector<int> first, last;
    std::vector<float> zmin_layer, zmax_layer;
    float XMin, XMax, YMin, YMax, ZMin, ZMax;
    std::vector<int> finish;
};

// ParallelMeshInit's type-R branch at one rank (src/CAinitialize.cpp:747-1003): bounds from every
// file, domain sizes, then the points of x/y range [2, nx-3] x [2, ny-3] (the one rank's range)
void mesh_reduced(Input &I, TemperatureGrid &T) {
    T.XMin = 1000000.0;
    T.YMin = 1000000.0;
    T.ZMin = 1000000.0;
    T.XMax = -1000000.0;
    T.YMax = -1000000.0;
    T.ZMax = -1000000.0;
    const int nfiles = (int)I.temp_paths.size(), L = I.layers;
    T.zmin_layer.assign(L, 0.0f);
    T.zmax_layer.assign(L, 0.0f);
    T.first.assign(L, 0);
    T.last.assign(L, 0);
    const int read = std::min(L, nfiles);
    for (int f = 1; f <= read; f++) {
        std::ifstream in(I.temp_paths[f - 1]);
        std::string line;
        std::getline(in, line);
        if (line.find("Number of temperature data points") != std::string::npos)
            throw std::runtime_error("oracle: old temperature format");
        double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300, z0 = 1e300, z1 = -1e300;
        while (std::getline(in, line) && !line.empty()) {
            std::vector<double> v = temperature_values(line, 3);
            x0 = std::min(x0, v[0]);
            x1 = std::max(x1, v[0]);
            y0 = std::min(y0, v[1]);
            y1 = std::max(y1, v[1]);
            z0 = std::min(z0, v[2]);
            z1 = std::max(z1, v[2]);
        }
        z0 += I.deltax * I.layer_height * (f - 1);
        z1 += I.deltax * I.layer_height * (f - 1);
        if (x0 < T.XMin)
            T.XMin = x0;
        if (x1 > T.XMax)
            T.XMax = x1;
        if (y0 < T.YMin)
            T.YMin = y0;
        if (y1 > T.YMax)
            T.YMax = y1;
        if (z0 < T.ZMin)
            T.ZMin = z0;
        if (z1 > T.ZMax)
            T.ZMax = z1;
        T.zmin_layer[f - 1] = z0;
        T.zmax_layer[f - 1] = z1;
    }
    for (int f = nfiles; f < L; f++) {
        if (nfiles == 1) {
            T.zmin_layer[f] = T.zmin_layer[f - 1] + I.deltax * I.layer_height;
            T.zmax_layer[f] = T.zmax_layer[f - 1] + I.deltax * I.layer_height;
        }
        else {
            int rep = f % nfiles, unit = f / nfiles;
            T.zmin_layer[f] = T.zmin_layer[rep] + unit * nfiles * I.deltax * I.layer_height;
            T.zmax_layer[f] = T.zmax_layer[rep] + unit * nfiles * I.deltax * I.layer_height;
        }
        T.ZMax += I.deltax * I.layer_height;
    }
    I.nx = round((T.XMax - T.XMin) / I.deltax) + 1 + 4;
    I.ny = round((T.YMax - T.YMin) / I.deltax) + 1 + 4;
    I.nz = round((T.ZMax - T.ZMin) / I.deltax) + 1 + 3;
    for (int f = 1; f <= read; f++) {
        std::ifstream in(I.temp_paths[f - 1]);
        std::string line;
        std::getline(in, line);
        T.first[f - 1] = (int)T.raw.size();
        while (std::getline(in, line) && !line.empty()) {
            std::vector<double> v = temperature_values(line, 6);
            int xi = round((v[0] - T.XMin) / I.deltax) + 2, yi = round((v[1] - T.YMin) / I.deltax) + 2;
            if (xi >= 2 && xi <= I.nx - 3 && yi >= 2 && yi <= I.ny - 3)
                T.raw.insert(T.raw.end(), v.begin(), v.end());
        }
        T.last[f - 1] = (int)T.raw.size();
    }
    for (int f = nfiles; f < L; f++) {
        int from = nfiles == 1 ? f - 1 : f % nfiles;
        T.first[f] = T.first[from];
        T.last[f] = T.last[from];
    }
}

// TempInit_Reduced at one rank (src/CAinitialize.cpp:1128-1405)
void temp_reduced(Input &I, TemperatureGrid &T, int MX, int MY, int nz, std::vector<int> &CTS, std::vector<float> &DU,
                  std::vector<int> &Layer, int &ZBound_High, int &nzActive) {
    double unrounded = I.ht_deltax / I.deltax, fl = floor(unrounded);
    if (unrounded - fl > 0.0005)
        throw std::runtime_error("oracle: temperature spacing not a multiple of the cell size");
    I.deltax = I.ht_deltax / fl;
    const int ratio = round(I.ht_deltax / I.deltax);
    const int lx = 2, ly = 2, ux = I.nx - 3, uy = I.ny - 3; // one rank: MyXOffset = MyYOffset = -1
    const int sx = ux - lx + 1, sy = uy - ly + 1;
    for (long p = 0; p < (long)MX * MY * nz; p++)
        Layer[p] = -1;
    T.finish.assign(I.layers, 0);
    for (int L = 0; L < I.layers; L++) {
        double small = 1000000000, large = 0;
        int nzt = round((T.zmax_layer[L] - T.zmin_layer[L]) / I.deltax) + 1;
        std::vector<std::vector<std::vector<double>>> CR(nzt, std::vector<std::vector<double>>(sx, std::vector<double>(sy, -1.0)));
        std::vector<std::vector<std::vector<double>>> TL = CR;
        int X = -1, Y = -1, Z = -1;
        for (int i = T.first[L]; i < T.last[L]; i++) {
            int pos = i % 6;
            if (pos == 0)
                X = round((T.raw[i] - T.XMin) / I.deltax) + 2;
            else if (pos == 1)
                Y = round((T.raw[i] - T.YMin) / I.deltax) + 2;
            else if (pos == 2)
                Z = round((T.raw[i] + I.deltax * I.layer_height * L - T.zmin_layer[L]) / I.deltax);
            else if (pos == 4) {
                if (T.raw[i] > TL.at(Z).at(X - lx).at(Y - ly)) {
                    TL[Z][X - lx][Y - ly] = T.raw[i];
                    if (T.raw[i] < small)
                        small = T.raw[i];
                }
                else
                    i = i + 1;
            }
            else if (pos == 5) {
                CR.at(Z).at(X - lx).at(Y - ly) = T.raw[i];
                float sol = TL[Z][X - lx][Y - ly] + I.freezing / CR[Z][X - lx][Y - ly];
                if (sol > large)
                    large = sol;
            }
        }
        T.finish[L] = round((large - small) / I.deltat);
        if (ratio != 1) {
            for (int k = 0; k < nzt; k++) {
                int LowZ = k - (k % ratio), HighZ = LowZ + ratio;
                double FHighZ = (double)(k - LowZ) / (double)(ratio), FLowZ = 1.0 - FHighZ;
                if (HighZ > nzt - 1)
                    HighZ = LowZ;
                for (int i = 0; i <= ux - lx; i++) {
                    int LowX = i - (i % ratio), HighX = LowX + ratio;
                    double FHighX = (double)(i - LowX) / (double)(ratio), FLowX = 1.0 - FHighX;
                    if (HighX >= ux - lx)
                        HighX = ux - lx;
                    for (int j = 0; j <= uy - ly; j++) {
                        int LowY = j - (j % ratio), HighY = LowY + ratio;
                        double FHighY = (float)(j - LowY) / (float)(ratio), FLowY = 1.0 - FHighY;
                        if (HighY >= uy - ly)
                            HighY = uy - ly;
                        for (auto *A : {&TL, &CR}) {
                            auto &V = *A;
                            double Pt1 = V[LowZ][LowX][LowY], Pt2 = V[LowZ][HighX][LowY];
                            double Pt12 = FLowX * Pt1 + FHighX * Pt2;
                            double Pt3 = V[LowZ][LowX][HighY], Pt4 = V[LowZ][HighX][HighY];
                            double Pt34 = FLowX * Pt3 + FHighX * Pt4;
                            double Pt1234 = Pt12 * FLowY + Pt34 * FHighY;
                            double Pt5 = V[HighZ][LowX][LowY], Pt6 = V[HighZ][HighX][LowY];
                            double Pt56 = FLowX * Pt5 + FHighX * Pt6;
                            double Pt7 = V[HighZ][LowX][HighY], Pt8 = V[HighZ][HighX][HighY];
                            double Pt78 = FLowX * Pt7 + FHighX * Pt8;
                            double Pt5678 = Pt56 * FLowY + Pt78 * FHighY;
                            if ((Pt1 > 0) && (Pt2 > 0) && (Pt3 > 0) && (Pt4 > 0) && (Pt5 > 0) && (Pt6 > 0) && (Pt7 > 0) &&
                                (Pt8 > 0))
                                V[k][i][j] = Pt1234 * FLowZ + Pt5678 * FHighZ;
                        }
                    }
                }
            }
        }
        if (L == 0) {
            ZBound_High = round((T.zmin_layer[0] - T.ZMin) / I.deltax) + 2 + nzt - 1;
            nzActive = ZBound_High + 1;
        }
        for (int k = 0; k < nzt; k++)
            for (int ii = lx; ii <= ux; ii++)
                for (int jj = ly; jj <= uy; jj++) {
                    double CTLiq = TL[k][ii - lx][jj - ly] - small;
                    if (CTLiq > 0) {
                        int ZOffset = round((T.zmin_layer[L] - T.ZMin) / I.deltax) + k + 2;
                        long p = (long)ZOffset * MX * MY + (long)(ii + 1) * MY + (jj + 1);
                        CTS.at(p) = round(CTLiq / I.deltat);
                        Layer[p] = L;
                        DU[p] = std::abs(CR[k][ii - lx][jj - ly]) * I.deltat;
                    }
                }
    }
}

// ---- state ---------------------------------------------------------------------------------------
struct Oracle {
    Input in;
    int MX, MY, nz, nzActive, ZBound_Low = 0, ZBound_High;
    int XOff = -1, YOff = -1;
    long N, NA;
    int NX[26], NY[26], NZ[26], ItList[9][26];
    std::vector<int> CellType, GrainID, CritTimeStep, LayerID;
    std::vector<float> UndercoolingChange, UndercoolingCurrent, DiagonalLength, DOCenter, CritDiagonalLength;
    std::vector<float> GrainUnitVector;
    std::vector<int> NucleiLocation, NucleationTimes;
    double A, B, C, D;
    int cycle = 0, nn = 0, layer = 0;
    bool layer_started = false; // the layer loop of oracle_run_to is inside layer `layer`
    std::vector<int> finish; // type R: per layer, FinishTimeStep
    std::vector<int> SteeringVector;
    // every census of the layer loop (oracle_run): cycle, superheated, undercooled, nucleation events,
    // remaining liquid, and the cycle jumped to (0: no jump)
    std::vector<std::array<long long, 6>> census;

    long idx(int k, int i, int j) const { return (long)k * MX * MY + (long)i * MY + j; }
};

// src/CAinitialize.cpp:595-745
void neighbour_tables(Oracle &o) {
    const int x[26] = {0, 1, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, 0, 1, -1, 0, 0, 1, -1, 1, -1};
    const int y[26] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};
    const int z[26] = {0, 0, 0, 1, -1, 1, 1, -1, -1, 1, -1, 1, 1, -1, -1, 0, 0, 0, 0, 0, 1, -1, 1, 1, -1, -1};
    for (int n = 0; n < 26; n++) {
        o.NX[n] = x[n];
        o.NY[n] = y[n];
        o.NZ[n] = z[n];
    }
    for (int c = 0; c < 9; c++) {
        int pos = 0;
        for (int n = 0; n < 26; n++) {
            bool keep;
            switch (c) {
            case 0: keep = true; break;
            case 1: keep = y[n] != -1; break;
            case 2: keep = y[n] != 1; break;
            case 3: keep = x[n] != -1; break;
            case 4: keep = x[n] != 1; break;
            case 5: keep = x[n] != -1 && y[n] != -1; break;
            case 6: keep = x[n] != 1 && y[n] != -1; break;
            case 7: keep = x[n] != -1 && y[n] != 1; break;
            default: keep = x[n] != 1 && y[n] != 1; break;
            }
            o.ItList[c][n] = 0;
            if (keep)
                o.ItList[c][pos++] = n;
        }
    }
}

// src/CAfunctions.cpp:169-213
int it_bounds(int RankX, int RankY, int MX, int MY) {
    if (RankY == 0)
        return RankX == 0 ? 5 : (RankX == MX - 1 ? 6 : 1);
    if (RankY == MY - 1)
        return RankX == 0 ? 7 : (RankX == MX - 1 ? 8 : 2);
    return RankX == 0 ? 3 : (RankX == MX - 1 ? 4 : 0);
}
int list_length(int b) { return b == 0 ? 26 : (b > 4 ? 11 : 17); }

// src/CAinitialize.cpp:1408-1441
void orientations(Oracle &o) {
    o.GrainUnitVector.assign(9 * NGrainOrientations, 0.0f);
    std::ifstream f(o.in.orientation_file);
    if (!f.is_open())
        throw std::runtime_error("cannot open " + o.in.orientation_file);
    std::string s;
    std::getline(f, s);
    for (int i = 0; i < NGrainOrientations; i++) {
        if (!std::getline(f, s))
            break;
        std::istringstream ss(s);
        int comp = 0, uv = 0;
        std::string t;
        while (ss && std::getline(ss, t, ',')) {
            o.GrainUnitVector[9 * i + 3 * uv + comp] = atof(t.c_str());
            if (++comp > 2) {
                comp = 0;
                uv++;
            }
        }
    }
}

// critical diagonal lengths of a fresh octahedron centred at the cell centre
// (src/CAupdate.cpp:112-194; src/CAinitialize.cpp:1963-2042)
void fresh_octahedron(Oracle &o, long D3D1, int GlobalX, int GlobalY, int GlobalZ, int MyGrainID) {
    o.DiagonalLength[D3D1] = 0.01;
    o.DOCenter[3 * D3D1] = GlobalX + 0.5;
    o.DOCenter[3 * D3D1 + 1] = GlobalY + 0.5;
    o.DOCenter[3 * D3D1 + 2] = GlobalZ + 0.5;
    int MyOrientation = ((abs(MyGrainID) - 1) % NGrainOrientations);
    const float *g = &o.GrainUnitVector[9 * MyOrientation];
    double xp = GlobalX + 0.5, yp = GlobalY + 0.5, zp = GlobalZ + 0.5;
    float cx = o.DOCenter[3 * D3D1], cy = o.DOCenter[3 * D3D1 + 1], cz = o.DOCenter[3 * D3D1 + 2];
    for (int n = 0; n < 26; n++) {
        double x0 = xp + o.NX[n] - cx;
        double y0 = yp + o.NY[n] - cy;
        double z0 = zp + o.NZ[n] - cz;
        double mag0 = pow(pow(x0, 2.0) + pow(y0, 2.0) + pow(z0, 2.0), 0.5);
        double d[3][3];
        for (int a = 0; a < 3; a++) {
            double ang = (g[3 * a] * x0 + g[3 * a + 1] * y0 + g[3 * a + 2] * z0) / mag0;
            for (int b = 0; b < 3; b++)
                d[a][b] = ang < 0 ? (double)g[3 * a + b] : (double)(-g[3 * a + b]);
        }
        double U1[3], U2[3];
        for (int b = 0; b < 3; b++) {
            U1[b] = d[1][b] - d[0][b];
            U2[b] = d[2][b] - d[0][b];
        }
        double UU0 = U1[1] * U2[2] - U1[2] * U2[1];
        double UU1 = U1[2] * U2[0] - U1[0] * U2[2];
        double UU2 = U1[0] * U2[1] - U1[1] * U2[0];
        double NDem = sqrt(UU0 * UU0 + UU1 * UU1 + UU2 * UU2);
        double n0 = UU0 / NDem, n1 = UU1 / NDem, n2 = UU2 / NDem;
        double ParaT = (n0 * x0 + n1 * y0 + n2 * z0) / (n0 * d[0][0] + n1 * d[0][1] + n2 * d[0][2]);
        float CDLVal = pow(pow(ParaT * d[0][0], 2.0) + pow(ParaT * d[0][1], 2.0) + pow(ParaT * d[0][2], 2.0), 0.5);
        o.CritDiagonalLength[26 * D3D1 + n] = CDLVal;
    }
}

void initialise(Oracle &o) {
    Input &I = o.in;
    neighbour_tables(o);
    TemperatureGrid T;
    if (I.type == "R")
        mesh_reduced(I, T);
    o.MX = I.nx + 2;
    o.MY = I.ny + 2;
    o.nz = I.nz;
    o.N = (long)o.MX * o.MY * o.nz;
    o.CritTimeStep.assign(o.N, 0);
    o.LayerID.assign(o.N, 0);
    o.UndercoolingChange.assign(o.N, 0.0f);
    o.UndercoolingCurrent.assign(o.N, 0.0f);
    o.CellType.assign(o.N, 0);
    o.GrainID.assign(o.N, 0);
    const int MX = o.MX, MY = o.MY, nz = o.nz;
    std::vector<int> seeds;
    if (I.type == "C") {
        // src/CAinitialize.cpp:1025-1055
        o.ZBound_High = nz - 1;
        o.nzActive = nz;
        for (int k = 0; k < nz; k++)
            for (int i = 0; i < MX; i++)
                for (int j = 0; j < MY; j++) {
                    long p = o.idx(k, i, j);
                    o.LayerID[p] = 0;
                    o.UndercoolingChange[p] = I.R * I.deltat;
                    o.CritTimeStep[p] = (int)(((k - 1) * I.G * I.deltax) / (I.R * I.deltat));
                }
    }
    else if (I.type == "R") {
        temp_reduced(I, T, MX, MY, nz, o.CritTimeStep, o.UndercoolingChange, o.LayerID, o.ZBound_High, o.nzActive);
        o.finish = T.finish;
    }
    else {
        // src/CAinitialize.cpp:1058-1124
        o.ZBound_High = I.spot_radius + 1;
        o.nzActive = I.spot_radius + 2;
        for (long p = 0; p < o.N; p++)
            o.LayerID[p] = -1;
        int nspots = I.nspx * I.nspy;
        float iso = (I.R / I.G) * I.deltat / I.deltax;
        int between = I.spot_radius / iso + (I.freezing / I.R) / I.deltat;
        // every layer's spots, later layers overwriting earlier ones
        for (int layer = 0; layer < I.layers; layer++)
            for (int n = 0; n < nspots; n++) {
                int xs = 2 + I.spot_radius + (n % I.nspx) * I.spot_offset;
                int ys = 2 + I.spot_radius + (n / I.nspx) * I.spot_offset;
                int zs = I.spot_radius + 2 + I.layer_height * layer;
                for (int k = 0; k < o.nzActive; k++) {
                    float dz = (float)(zs - (k + I.layer_height * layer));
                    for (int i = 0; i < MX; i++) {
                        float dx = (float)(xs - (i + o.XOff));
                        for (int j = 0; j < MY; j++) {
                            float dy = (float)(ys - (j + o.YOff));
                            float d = sqrtf(dx * dx + dy * dy + dz * dz);
                            if (d <= I.spot_radius) {
                                long p = o.idx(k + layer * I.layer_height, i, j);
                                o.CritTimeStep[p] = 1 + (int)(((float)(I.spot_radius) - d) / iso) + between * n;
                                o.UndercoolingChange[p] = I.R * I.deltat;
                                o.LayerID[p] = layer;
                            }
                        }
                    }
                }
            }
    }
    o.NA = (long)MX * MY * o.nzActive;
    o.DiagonalLength.assign(o.NA, 0.0f);
    o.DOCenter.assign(3 * o.NA, 0.0f);
    o.CritDiagonalLength.assign(26 * o.NA, 0.0f);
    orientations(o);
    const int nxg = I.nx, nyg = I.ny;
    auto is_wall = [&](int i, int j, int k) {
        int gx = i + o.XOff, gy = j + o.YOff;
        return gx == -1 || gx == nxg || gy == -1 || gy == nyg || k == 0 || k == nz - 1;
    };
    if (I.type == "C") {
        // src/CAinitialize.cpp:1460-1529
        std::mt19937_64 gen(0);
        std::uniform_real_distribution<double> dis(0.0, 1.0);
        for (int k = 0; k < nz; k++)
            for (int i = 0; i < MX; i++)
                for (int j = 0; j < MY; j++) {
                    long p = o.idx(k, i, j);
                    if (is_wall(i, j, k)) {
                        o.CellType[p] = Wall;
                        o.GrainID[p] = 0;
                    }
                    else if (k == 1 && i > 0 && i < MX - 1 && j > 0 && j < MY - 1) {
                        double R = dis(gen);
                        o.CellType[p] = R < I.fract ? Active : Liquid;
                    }
                    else
                        o.CellType[p] = Liquid;
                }
        int id = 1;
        for (long p = 0; p < o.N; p++)
            if (o.CellType[p] == Active)
                o.GrainID[p] = id++;
    }
    else {
        // src/CAinitialize.cpp:1597-1732
        std::mt19937_64 gen(1.0);
        std::uniform_real_distribution<double> dis(0.0, 1.0);
        float sp = I.grain_spacing;
        double prob = (I.deltax * I.deltax * I.deltax) / (sp * sp * sp * pow(10, -18));
        for (int k = 1; k <= o.nzActive; k++)
            for (int i = 1; i < nxg - 1; i++)
                for (int j = 1; j < nyg - 1; j++)
                    if (dis(gen) < prob) {
                        seeds.push_back(i);
                        seeds.push_back(j);
                        seeds.push_back(k);
                    }
        int ns = (int)seeds.size() / 3;
        for (int k = 1; k < o.nzActive; k++)
            for (int i = 0; i < MX; i++)
                for (int j = 0; j < MY; j++) {
                    long p = o.idx(k, i, j);
                    if (o.CritTimeStep[p] == 0) {
                        float mind = (float)(o.NA);
                        int best = -1;
                        for (int s = 0; s < ns; s++) {
                            float ddx = (float)(abs(seeds[3 * s] - (i + o.XOff)));
                            float ddy = (float)(abs(seeds[3 * s + 1] - (j + o.YOff)));
                            float ddz = (float)(abs(seeds[3 * s + 2] - k));
                            float d = sqrtf(ddx * ddx + ddy * ddy + ddz * ddz);
                            if (d < mind) {
                                best = s;
                                mind = d;
                            }
                        }
                        o.GrainID[p] = best + 1;
                    }
                    else
                        o.GrainID[p] = 0;
                }
        for (int k = o.nzActive; k < nz; k++)
            for (int i = 1; i < MX - 1; i++)
                for (int j = 1; j < MY - 1; j++)
                    if (o.CritTimeStep[o.idx(k, i, j)] != 0)
                        o.GrainID[o.idx(k, i, j)] = 0;
        int id = ns + 1;
        for (long p = (long)MX * MY * o.nzActive; p < o.N; p++)
            if (o.CritTimeStep[p] == 0)
                o.GrainID[p] = id++;
        // src/CAinitialize.cpp:1736-1830 (with the extra wall ring of type R inputs that ask for it)
        for (int k = 0; k < nz; k++)
            for (int i = 0; i < MX; i++)
                for (int j = 0; j < MY; j++) {
                    const int gx = i + o.XOff, gy = j + o.YOff;
                    const bool extra = I.extra_walls && (gx == 0 || gx == nxg - 1 || gy == 0 || gy == nyg - 1 ||
                                                         gx == 1 || gx == nxg - 2 || gy == 1 || gy == nyg - 2);
                    if (is_wall(i, j, k) || extra) {
                        o.CellType[o.idx(k, i, j)] = Wall;
                        o.GrainID[o.idx(k, i, j)] = 0;
                    }
                }
        for (int k = 1; k < nz - 1; k++)
            for (int j = 0; j < MY; j++)
                for (int i = 0; i < MX; i++)
                    o.CellType[o.idx(k, i, j)] = o.CritTimeStep[o.idx(k, i, j)] == 0 ? Solid : Liquid;
        for (int k = 1; k < nz - 1; k++)
            for (int j = 0; j < MY; j++)
                for (int i = 0; i < MX; i++) {
                    long p = o.idx(k, i, j);
                    if (o.CritTimeStep[p] != 0)
                        continue;
                    int b = it_bounds(i, j, MX, MY);
                    for (int ll = 0; ll < list_length(b); ll++) {
                        int l = o.ItList[b][ll];
                        long q = o.idx(k + o.NZ[l], i + o.NX[l], j + o.NY[l]);
                        if (o.CritTimeStep[q] > 0 && o.CellType[q] != Wall) {
                            o.CellType[p] = Active;
                            o.UndercoolingChange[p] = o.UndercoolingChange[q];
                            break;
                        }
                    }
                }
    }
    // src/CAinitialize.cpp:1834-2206 (one rank)
    {
        std::mt19937_64 gen(0);
        std::uniform_real_distribution<double> dis(0.0, 1.0);
        double prob = I.NMax * I.deltax * I.deltax * I.deltax;
        for (int k = 1; k < nz - 1; k++)
            for (int j = 1; j < MY - 1; j++)
                for (int i = 1; i < MX - 1; i++) {
                    long p = o.idx(k, i, j);
                    if (o.CritTimeStep[p] != 0 && dis(gen) < prob)
                        o.CellType[p] = TemporaryInit;
                }
        int NCounter = -1;
        for (int k = 1; k < nz - 1; k++)
            for (int i = 0; i < MX; i++)
                for (int j = 0; j < MY; j++) {
                    long p = o.idx(k, i, j);
                    if (o.CellType[p] == Active) {
                        if (k <= o.ZBound_High)
                            fresh_octahedron(o, p - (long)o.ZBound_Low * MX * MY, i + o.XOff, j + o.YOff, k,
                                             o.GrainID[p]);
                    }
                    else if (o.CellType[p] == TemporaryInit) {
                        o.GrainID[p] = NCounter--;
                    }
                }
        for (int k = 1; k < nz - 1; k++)
            for (int i = 1; i < MX - 1; i++)
                for (int j = 1; j < MY - 1; j++) {
                    long p = o.idx(k, i, j);
                    if (o.CellType[p] != Liquid)
                        continue;
                    int b = it_bounds(i, j, MX, MY), LCount = 0;
                    for (int ll = 0; ll < list_length(b); ll++) {
                        int l = o.ItList[b][ll];
                        int t = o.CellType[o.idx(k + o.NZ[l], i + o.NX[l], j + o.NY[l])];
                        if (t != Solid && t != Wall)
                            LCount++;
                    }
                    if (LCount == 0)
                        o.CellType[p] = Solid;
                }
    }
    // src/CAinitialize.cpp:2213-2247, 2758-2768
    {
        std::default_random_engine generator;
        std::normal_distribution<double> distribution(I.dTN, I.dTsigma);
        for (long p = 0; p < o.N; p++)
            if (o.CellType[p] == TemporaryInit) {
                o.NucleiLocation.push_back((int)p);
                double und = distribution(generator);
                int t = o.CritTimeStep[p] + round(und / o.UndercoolingChange[p]);
                o.NucleationTimes.push_back(std::max(o.CritTimeStep[p], t));
                o.CellType[p] = Liquid;
            }
    }
    // src/runCA.cpp:198-200
    o.A = I.A * I.deltat / I.deltax;
    o.B = I.B * I.deltat / I.deltax;
    o.C = I.C * I.deltat / I.deltax;
    o.D = I.D;
    o.SteeringVector.resize(o.NA);
}

// ---- one cycle ----------------------------------------------------------------------------------
// src/CAupdate.cpp:67-200
void nucleation(Oracle &o) {
    const int MX = o.MX, MY = o.MY;
    for (size_t n = 0; n < o.NucleiLocation.size(); n++) {
        long g = o.NucleiLocation[n];
        if (o.cycle >= o.NucleationTimes[n] && o.CellType[g] == Liquid && o.LayerID[g] <= o.layer) {
            o.CellType[g] = TemporaryUpdate;
            int GlobalZ = g / (MX * MY);
            int Rem = g % (MX * MY);
            int RankX = Rem / MY, RankY = Rem % MY;
            if (RankX > 0 && RankX < MX - 1 && RankY > 0 && RankY < MY - 1)
                o.nn++;
            long D3D1 = (long)(GlobalZ - o.ZBound_Low) * MX * MY + (long)RankX * MY + RankY;
            fresh_octahedron(o, D3D1, RankX + o.XOff, RankY + o.YOff, GlobalZ, o.GrainID[g]);
            o.CellType[g] = Active;
        }
    }
}

// capture of neighbour l of active cell D3D1 (src/CAupdate.cpp:353-563)
void capture(Oracle &o, long D3D1, long Nb, long GlobalNb, int RankX, int RankY, int GlobalZ, int l) {
    const float *g;
    int GlobalX = RankX + o.XOff, GlobalY = RankY + o.YOff;
    long Global = D3D1 + (long)o.ZBound_Low * o.MX * o.MY;
    int h = o.GrainID[Global];
    int MyOrientation = ((abs(h) - 1) % NGrainOrientations);
    g = &o.GrainUnitVector[9 * MyOrientation];
    o.GrainID[GlobalNb] = h;
    double cxold = o.DOCenter[3 * D3D1], cyold = o.DOCenter[3 * D3D1 + 1], czold = o.DOCenter[3 * D3D1 + 2];
    double xp = GlobalX + o.NX[l] + 0.5;
    double yp = GlobalY + o.NY[l] + 0.5;
    double zp = GlobalZ + o.NZ[l] + 0.5;
    double x0 = xp - cxold, y0 = yp - cyold, z0 = zp - czold;
    double mag0 = sqrtf(x0 * x0 + y0 * y0 + z0 * z0);
    double Angle1 = (g[0] * x0 + g[1] * y0 + g[2] * z0) / mag0;
    double Angle2 = (g[3] * x0 + g[4] * y0 + g[5] * z0) / mag0;
    double Angle3 = (g[6] * x0 + g[7] * y0 + g[8] * z0) / mag0;
    double Diag1X = g[0] * (2 * (Angle1 < 0) - 1), Diag1Y = g[1] * (2 * (Angle1 < 0) - 1),
           Diag1Z = g[2] * (2 * (Angle1 < 0) - 1);
    double Diag2X = g[3] * (2 * (Angle2 < 0) - 1), Diag2Y = g[4] * (2 * (Angle2 < 0) - 1),
           Diag2Z = g[5] * (2 * (Angle2 < 0) - 1);
    double Diag3X = g[6] * (2 * (Angle3 < 0) - 1), Diag3Y = g[7] * (2 * (Angle3 < 0) - 1),
           Diag3Z = g[8] * (2 * (Angle3 < 0) - 1);
    double U1[3] = {Diag2X - Diag1X, Diag2Y - Diag1Y, Diag2Z - Diag1Z};
    double U2[3] = {Diag3X - Diag1X, Diag3Y - Diag1Y, Diag3Z - Diag1Z};
    double UU[3] = {U1[1] * U2[2] - U1[2] * U2[1], U1[2] * U2[0] - U1[0] * U2[2], U1[0] * U2[1] - U1[1] * U2[0]};
    double NDem = sqrtf(UU[0] * UU[0] + UU[1] * UU[1] + UU[2] * UU[2]);
    double nrm[3] = {UU[0] / NDem, UU[1] / NDem, UU[2] / NDem};
    double ParaT = (nrm[0] * x0 + nrm[1] * y0 + nrm[2] * z0) / (nrm[0] * Diag1X + nrm[1] * Diag1Y + nrm[2] * Diag1Z);
    double TX[3] = {cxold + ParaT * Diag1X, cxold + ParaT * Diag2X, cxold + ParaT * Diag3X};
    double TY[3] = {cyold + ParaT * Diag1Y, cyold + ParaT * Diag2Y, cyold + ParaT * Diag3Y};
    double TZ[3] = {czold + ParaT * Diag1Z, czold + ParaT * Diag2Z, czold + ParaT * Diag3Z};
    double Dist[3];
    for (int q = 0; q < 3; q++)
        Dist[q] = sqrtf(((TX[q] - xp) * (TX[q] - xp)) + ((TY[q] - yp) * (TY[q] - yp)) + ((TZ[q] - zp) * (TZ[q] - zp)));
    int x = (Dist[0] < Dist[1]), y = (Dist[1] < Dist[2]), z = (Dist[2] < Dist[0]);
    int idx = 2 * (z - y) * z + (y - x) * y;
    double mind = Dist[idx], xc = TX[idx], yc = TY[idx], zc = TZ[idx];
    double x1 = TX[(idx + 1) % 3], y1 = TY[(idx + 1) % 3], z1 = TZ[(idx + 1) % 3];
    double x2 = TX[(idx + 2) % 3], y2 = TY[(idx + 2) % 3], z2 = TZ[(idx + 2) % 3];
    double D1 = sqrtf(((xp - x2) * (xp - x2)) + ((yp - y2) * (yp - y2)) + ((zp - z2) * (zp - z2)));
    double D2 = sqrtf(((xc - x2) * (xc - x2)) + ((yc - y2) * (yc - y2)) + ((zc - z2) * (zc - z2)));
    double D3 = sqrtf(((xp - x1) * (xp - x1)) + ((yp - y1) * (yp - y1)) + ((zp - z1) * (zp - z1)));
    double D4 = sqrtf(((xc - x1) * (xc - x1)) + ((yc - y1) * (yc - y1)) + ((zc - z1) * (zc - z1)));
    double I1 = 0, I2 = D2, J1 = 0, J2 = D4;
    if (mind != 0) {
        I1 = D1 * ((xp - x2) * (xc - x2) + (yp - y2) * (yc - y2) + (zp - z2) * (zc - z2)) / (D1 * D2);
        I2 = D2 - I1;
        J1 = D3 * ((xp - x1) * (xc - x1) + (yp - y1) * (yc - y1) + (zp - z1) * (zc - z1)) / (D3 * D4);
        J2 = D4 - J1;
    }
    double L12 = 0.5 * (std::min(I1, sqrt(3.0)) + std::min(I2, sqrt(3.0)));
    double L13 = 0.5 * (std::min(J1, sqrt(3.0)) + std::min(J2, sqrt(3.0)));
    double NewODiagL = sqrt(2.0) * std::max(L12, L13);
    o.DiagonalLength[Nb] = NewODiagL;
    double CD[3] = {xc - cxold, yc - cyold, zc - czold};
    double nd = sqrt(CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2]);
    double cx = xc - NewODiagL * (CD[0] / nd);
    double cy = yc - NewODiagL * (CD[1] / nd);
    double cz = zc - NewODiagL * (CD[2] / nd);
    o.DOCenter[3 * Nb] = cx;
    o.DOCenter[3 * Nb + 1] = cy;
    o.DOCenter[3 * Nb + 2] = cz;
    double Fx[4] = {g[0] + g[3] + g[6], g[0] - g[3] + g[6], g[0] + g[3] - g[6], g[0] - g[3] - g[6]};
    double Fy[4] = {g[1] + g[4] + g[7], g[1] - g[4] + g[7], g[1] + g[4] - g[7], g[1] - g[4] - g[7]};
    double Fz[4] = {g[2] + g[5] + g[8], g[2] - g[5] + g[8], g[2] + g[5] - g[8], g[2] - g[5] - g[8]};
    for (int n = 0; n < 26; n++) {
        double a0 = xp + o.NX[n] - cx, b0 = yp + o.NY[n] - cy, c0 = zp + o.NZ[n] - cz;
        double Dv[4];
        for (int f = 0; f < 4; f++)
            Dv[f] = a0 * Fx[f] + b0 * Fy[f] + c0 * Fz[f];
        double m = std::max(std::max(fabs(Dv[0]), fabs(Dv[1])), std::max(fabs(Dv[2]), fabs(Dv[3])));
        o.CritDiagonalLength[26 * Nb + n] = m;
    }
}

// src/CAupdate.cpp:204-728 with the Serial backend's ascending order
// First pass of CellCapture (src/CAupdate.cpp:217-242) over window cells [lo, hi): undercooling
// update, and the active cells listed in ascending order. Cells are independent in this pass, so
// contiguous ranges may run on separate threads; their lists, joined in range order, are the Serial
// backend's steering vector.
int pass1_range(Oracle &o, long lo, long hi, int *steer) {
    // the window index D3D1 maps to the global index D3D1 + ZBound_Low * MX * MY
    const long shift = (long)o.ZBound_Low * o.MX * o.MY;
    const int *ctype = o.CellType.data() + shift, *layer = o.LayerID.data() + shift,
              *cts = o.CritTimeStep.data() + shift;
    float *u = o.UndercoolingCurrent.data() + shift;
    const float *du = o.UndercoolingChange.data() + shift;
    const int lay = o.layer, cycle = o.cycle;
    int n = 0;
    for (long D3D1 = lo; D3D1 < hi; D3D1++) {
        int ct = ctype[D3D1];
        if (layer[D3D1] <= lay && ct != Solid && cycle > cts[D3D1]) {
            u[D3D1] += du[D3D1] * ((ct == Liquid) + (ct == Active));
            if (ct == Active)
                steer[n++] = (int)D3D1;
        }
    }
    return n;
}

void cell_capture(Oracle &o) {
    const int MX = o.MX, MY = o.MY;
    int numSteer = 0;
    if (g_threads <= 1) {
        numSteer = pass1_range(o, 0, o.NA, o.SteeringVector.data());
    }
    else {
        // range t lists into SteeringVector from its own start lo_t (a range lists at most its own
        // cells), then the lists are moved down to be contiguous, in range order
        const int T = g_threads;
        std::vector<int> count(T);
#pragma omp parallel for num_threads(T) schedule(static, 1)
        for (int t = 0; t < T; t++) {
            const long lo = o.NA * t / T, hi = o.NA * (t + 1) / T;
            count[t] = pass1_range(o, lo, hi, o.SteeringVector.data() + lo);
        }
        for (int t = 0; t < T; t++) {
            const long lo = o.NA * t / T;
            std::memmove(o.SteeringVector.data() + numSteer, o.SteeringVector.data() + lo, sizeof(int) * count[t]);
            numSteer += count[t];
        }
    }
    for (int num = 0; num < numSteer; num++) {
        long D3D1 = o.SteeringVector[num];
        int RankZ = D3D1 / (MX * MY);
        int Rem = D3D1 % (MX * MY);
        int RankX = Rem / MY, RankY = Rem % MY;
        int GlobalZ = RankZ + o.ZBound_Low;
        long Global = (long)GlobalZ * MX * MY + Rem;
        double LocU = o.UndercoolingCurrent[Global];
        LocU = std::min(210.0, LocU);
        double V = o.A * pow(LocU, 3.0) + o.B * pow(LocU, 2.0) + o.C * LocU + o.D;
        V = std::max(0.0, V);
        o.DiagonalLength[D3D1] += std::min(0.045, V);
        int LCount = 0;
        int b = it_bounds(RankX, RankY, MX, MY);
        for (int ll = 0; ll < list_length(b); ll++) {
            int l = o.ItList[b][ll];
            int nX = RankX + o.NX[l], nY = RankY + o.NY[l], nZ = RankZ + o.NZ[l];
            if (nZ < o.nzActive) {
                long Nb = (long)nZ * MX * MY + (long)nX * MY + nY;
                long GNb = (long)(nZ + o.ZBound_Low) * MX * MY + (long)nX * MY + nY;
                if (o.CellType[GNb] == Liquid)
                    LCount = 1;
                if (o.DiagonalLength[D3D1] >= o.CritDiagonalLength[26 * D3D1 + l] && o.CellType[GNb] == Liquid) {
                    o.CellType[GNb] = TemporaryUpdate;
                    capture(o, D3D1, Nb, GNb, RankX, RankY, GlobalZ, l);
                    o.CellType[GNb] = Active;
                }
            }
        }
        if (LCount == 0)
            o.CellType[Global] = Solid;
    }
}

// src/CAupdate.cpp:732-822 (one rank): returns XSwitch
int check(Oracle &o) {
    unsigned long sh = 0, uc = 0;
    for (long p = 0; p < o.N; p++)
        if (o.LayerID[p] == o.layer && o.CellType[p] == Liquid) {
            if (o.CritTimeStep[p] > o.cycle)
                sh++;
            else
                uc++;
        }
    unsigned long rem = 0;
    for (long p = 0; p < o.N; p++)
        if (o.LayerID[p] != o.layer && o.CellType[p] == Liquid)
            rem++;
    o.census.push_back({(long long)o.cycle, (long long)sh, (long long)uc, (long long)o.nn, (long long)rem, 0});
    if (sh + uc == 0)
        return 1;
    if ((o.in.type == "S" || o.in.type == "R") && uc == 0) {
        unsigned long next = (unsigned long)-1;
        for (long D3D1 = 0; D3D1 < o.NA; D3D1++) {
            long g = D3D1 + (long)o.ZBound_Low * o.MX * o.MY;
            unsigned long cts = (unsigned long)(o.CritTimeStep[g]);
            if (o.CellType[g] == Liquid && o.LayerID[g] == o.layer && cts < next)
                next = cts;
        }
        if ((next - o.cycle) > 5000) {
            o.cycle = next - 1;
            o.census.back()[5] = (long long)next;
        }
        // src/CAupdate.cpp:818-819
        if (o.in.type == "R" && o.cycle >= o.finish[o.layer])
            return 1;
    }
    return 0;
}

// src/CAinitialize.cpp:2772-2837 (one rank): the window's new bottom is one plane below the lowest
// active cell, its new top the highest cell of the next layer
void domain_shift_and_resize(Oracle &o) {
    int lo = INT_MAX, hi = INT_MIN;
    const long plane = (long)o.MX * o.MY;
    for (long p = 0; p < o.N; p++) {
        int z = (int)(p / plane);
        if (o.CellType[p] == Active && z < lo)
            lo = z;
        if (o.LayerID[p] == o.layer + 1 && z > hi)
            hi = z;
    }
    o.ZBound_Low = lo - 1;
    o.ZBound_High = hi;
    o.nzActive = o.ZBound_High - o.ZBound_Low + 1;
    o.NA = plane * o.nzActive;
}

// src/CAinitialize.cpp:2840-2982: window arrays zeroed, fresh octahedra for the window's active cells
void layer_setup(Oracle &o) {
    const int MX = o.MX, MY = o.MY;
    o.DiagonalLength.assign(o.NA, 0.0f);
    o.DOCenter.assign(3 * o.NA, 0.0f);
    o.CritDiagonalLength.assign(26 * o.NA, 0.0f);
    o.SteeringVector.assign(o.NA, 0);
    for (long D3D1 = 0; D3D1 < o.NA; D3D1++) {
        int RankZ = D3D1 / (MX * MY);
        int Rem = D3D1 % (MX * MY);
        int RankX = Rem / MY, RankY = Rem % MY;
        int GlobalZ = RankZ + o.ZBound_Low;
        long g = (long)GlobalZ * MX * MY + Rem;
        if (o.CellType[g] == Active)
            fresh_octahedron(o, D3D1, RankX + o.XOff, RankY + o.YOff, GlobalZ, o.GrainID[g]);
    }
}

} // namespace

extern "C" {

const char *oracle_error(void) { return g_error.c_str(); }

void *oracle_create(const char *input_file, const char *data_dir) {
    try {
        Oracle *o = new Oracle();
        o->in = read_input(input_file, data_dir);
        initialise(*o);
        return o;
    }
    catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

void oracle_free(void *p) { delete static_cast<Oracle *>(p); }

int oracle_geometry(void *p, long long *out) {
    Oracle &o = *static_cast<Oracle *>(p);
    out[0] = o.MX;
    out[1] = o.MY;
    out[2] = o.nz;
    out[3] = o.nzActive;
    out[4] = o.N;
    out[5] = o.NA;
    return 0;
}

// n raw cycles: cycle++, Nucleation, CellCapture (src/runCA.cpp:291-311), no termination check
int oracle_step(void *p, int n) {
    Oracle &o = *static_cast<Oracle *>(p);
    for (int q = 0; q < n; q++) {
        o.cycle++;
        nucleation(o);
        cell_capture(o);
    }
    return 0;
}

// src/runCA.cpp:282-411: every layer's cycles, the window moved between layers. Stops early (returns
// 1) once a cycle equal to stop_cycle has run; a later call resumes the same layer loop.
int oracle_run_to(void *p, int stop_cycle, int *final_cycle) {
    Oracle &o = *static_cast<Oracle *>(p);
    for (; o.layer < o.in.layers; o.layer++) {
        if (!o.layer_started) {
            o.nn = 0;
            o.layer_started = true;
        }
        int XSwitch = 0;
        do {
            o.cycle++;
            nucleation(o);
            cell_capture(o);
            if (o.cycle % 1000 == 0)
                XSwitch = check(o);
            if (XSwitch == 0 && o.cycle == stop_cycle) {
                *final_cycle = o.cycle;
                return 1;
            }
        } while (XSwitch == 0);
        o.layer_started = false;
        if (o.layer != o.in.layers - 1) {
            domain_shift_and_resize(o);
            layer_setup(o);
            o.cycle = 0;
        }
    }
    o.layer = o.in.layers - 1;
    *final_cycle = o.cycle;
    return 0;
}

int oracle_run(void *p, int *final_cycle) { return oracle_run_to(p, INT_MIN, final_cycle); }

int oracle_cycle(void *p) { return static_cast<Oracle *>(p)->cycle; }

// host threads of CellCapture's dense first pass (results do not depend on it)
void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

// the censuses of oracle_run so far, 6 numbers each (cycle, superheated, undercooled, nucleation
// events, remaining liquid, cycle jumped to or 0); copies up to max of them, returns how many exist
int oracle_census(void *p, long long *out, int max) {
    Oracle &o = *static_cast<Oracle *>(p);
    for (int q = 0; q < max && q < (int)o.census.size(); q++)
        for (int f = 0; f < 6; f++)
            out[6 * q + f] = o.census[q][f];
    return (int)o.census.size();
}

int oracle_fields(void *p, int *cell_type, int *grain_id, float *dl, float *doc, float *cdl) {
    Oracle &o = *static_cast<Oracle *>(p);
    if (cell_type)
        std::memcpy(cell_type, o.CellType.data(), o.N * 4);
    if (grain_id)
        std::memcpy(grain_id, o.GrainID.data(), o.N * 4);
    if (dl)
        std::memcpy(dl, o.DiagonalLength.data(), o.NA * 4);
    if (doc)
        std::memcpy(doc, o.DOCenter.data(), o.NA * 12);
    if (cdl)
        std::memcpy(cdl, o.CritDiagonalLength.data(), o.NA * 104);
    return 0;
}

} // extern "C"
