// Test infrastructure only: a serial CPU restatement of the ExaCA reference's per-cycle update and
// of the initialisation it needs, used by the tests as the checker of the CUDA solver. It is never
// linked into or called by the product.
//
// Parity: pinned. tests/test_oracle.py checks this restatement bit for bit against the final
// GrainID / CellType arrays, final cycle and post-init fields of the reference itself (compiled
// from its unmodified sources against single-rank shims), stored in tests/golden/*.npz.
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
//   int  oracle_run(void *o, int *final_cycle)          to termination of the last layer, as
//                                                      RunProgram_Reduced does
//   int  oracle_cycle(void *o)
//   int  oracle_fields(void *o, int *cell_type, int *grain_id, float *dl, float *doc, float *cdl)
//   void oracle_free(void *o)
#include <algorithm>
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

// ---- input file (src/CAinitialize.cpp:24-576, the C and S branches) --------------------------
struct Input {
    std::string type;
    double A, B, C, D, freezing;
    double deltax, NMax, dTN, dTsigma, deltat, G, R, fract;
    int nx, ny, nz, nspx, nspy, spot_offset, spot_radius, layers, layer_height;
    float grain_spacing;
    std::string orientation_file;
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
    // key check by substring; the value is everything after the colon, whitespace removed
    std::string value(const std::string &key) {
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
            if (k.find(key) == std::string::npos)
                throw std::runtime_error("expected key " + key);
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
    else {
        throw std::runtime_error("oracle: problem types C and S only");
    }
    return I;
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
    std::vector<int> SteeringVector;

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
    const Input &I = o.in;
    neighbour_tables(o);
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
        // src/CAinitialize.cpp:1736-1830
        for (int k = 0; k < nz; k++)
            for (int i = 0; i < MX; i++)
                for (int j = 0; j < MY; j++)
                    if (is_wall(i, j, k)) {
                        o.CellType[o.idx(k, i, j)] = Wall;
                        o.GrainID[o.idx(k, i, j)] = 0;
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
void cell_capture(Oracle &o) {
    const int MX = o.MX, MY = o.MY;
    int numSteer = 0;
    for (long D3D1 = 0; D3D1 < o.NA; D3D1++) {
        int RankZ = D3D1 / (MX * MY);
        int Rem = D3D1 % (MX * MY);
        long Global = (long)(RankZ + o.ZBound_Low) * MX * MY + Rem;
        int ct = o.CellType[Global];
        if (o.LayerID[Global] <= o.layer && ct != Solid && o.cycle > o.CritTimeStep[Global]) {
            o.UndercoolingCurrent[Global] += o.UndercoolingChange[Global] * ((ct == Liquid) + (ct == Active));
            if (ct == Active)
                o.SteeringVector[numSteer++] = (int)D3D1;
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
    if (sh + uc == 0)
        return 1;
    if (o.in.type == "S" && uc == 0) {
        unsigned long next = (unsigned long)-1;
        for (long D3D1 = 0; D3D1 < o.NA; D3D1++) {
            long g = D3D1 + (long)o.ZBound_Low * o.MX * o.MY;
            unsigned long cts = (unsigned long)(o.CritTimeStep[g]);
            if (o.CellType[g] == Liquid && o.LayerID[g] == o.layer && cts < next)
                next = cts;
        }
        if ((next - o.cycle) > 5000)
            o.cycle = next - 1;
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

// src/runCA.cpp:282-411: every layer's cycles, the window moved between layers
int oracle_run(void *p, int *final_cycle) {
    Oracle &o = *static_cast<Oracle *>(p);
    for (; o.layer < o.in.layers; o.layer++) {
        int XSwitch = 0;
        o.nn = 0;
        do {
            o.cycle++;
            nucleation(o);
            cell_capture(o);
            if (o.cycle % 1000 == 0)
                XSwitch = check(o);
        } while (XSwitch == 0);
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

int oracle_cycle(void *p) { return static_cast<Oracle *>(p)->cycle; }

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
