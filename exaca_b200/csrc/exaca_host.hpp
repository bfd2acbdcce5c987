// Host-side data model of one ExaCA problem (one domain) for the B200 solver.
//
// The reference keeps this state in ~20 Kokkos views owned by RunProgram_Reduced
// (src/runCA.cpp:19-256). Here it is one Problem object: parsed inputs, the single-rank geometry,
// and the initialised fields that are uploaded once to a device pool slot.
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>
#include "directions.hpp"

namespace exaca {

// Cell types, same numbering as the reference enum TypeNames (src/CAtypes.hpp:11).
enum CellTypeCode : int8_t {
    kWall = 0,
    kSolid = 1,
    kActive = 2,
    kTemporaryUpdate = 3,
    kTemporaryInit = 4,
    kLiquid = 5,
    kGhost = 6
};

constexpr int kNumOrientations = 10000; // src/runCA.cpp:133

// A valid input this solver does not handle (substrate files, more than 127 layers, more distinct
// UndercoolingChange values than the growth tables hold).
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// The HBM budget or slot table of a pool cannot take a problem.
struct AdmissionRefused : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// A CUDA runtime error or a device-side error flag.
struct DeviceError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Every value the reference reads from an input file and its material file
// (src/CAinitialize.cpp:232-576). Units follow the reference: deltax and deltat in SI.
struct InputConfig {
    std::string input_file;
    std::string simulation_type; // "C", "S" or "R"
    int decomposition_strategy = 1;
    std::string material_name;
    double A = 0, B = 0, C = 0, D = 0, freezing_range = 0;
    double deltax = 0;  // m
    double nread = 0;   // nucleation density / 1e12
    double nmax = 0;    // m^-3
    double dTN = 0, dTsigma = 0;
    std::string path_to_output, output_file;
    std::string orientation_file; // resolved path
    // type R (temperature data from files)
    double ht_deltax = 0;
    std::string temppath, tempfile;
    int temp_files_in_series = 0;
    bool extra_walls = false;
    bool remelting = false;
    // time step and layers
    double deltat = 0;
    int number_of_layers = 1, layer_height = 0;
    // substrate (S/R)
    std::string substrate_file_name;
    float substrate_grain_spacing = 0.0f;
    bool use_substrate_file = false;
    // C and S
    double G = 0, R = 0;
    int nx = 0, ny = 0, nz = 0;
    double fract_surface_sites_active = 0;
    int nspots_x = 0, nspots_y = 0, spot_offset = 0, spot_radius = 0;
    // outputs
    int print_debug = 0;
    bool print_misorientation = false, print_full_output = false;
};

// Single-rank decomposition (src/CAfunctions.cpp:34-166 at np = 1): one ghost/wall ring in x and y.
struct Geometry {
    int nx = 0, ny = 0, nz = 0; // global sizes, wall layers included
    int mx = 0, my = 0;         // MyXSlices, MyYSlices
    int xoff = 0, yoff = 0;     // MyXOffset, MyYOffset
    int nz_active = 0, zbound_low = 0, zbound_high = 0;
    long domain_size = 0; // mx * my * nz
    long active_size = 0; // mx * my * nz_active
    int procs_x = 1, procs_y = 1;
};

// What the per-cell fields of a type-C problem are made of: they are written on the device at
// admission (src/CAinitialize.cpp:1025-1055, 1460-1529, 1834-2206 as one pass over the cells plus
// the scatter of the seeds and nuclei), and on the host only when a caller asks for them.
struct DirectionalSeeds {
    bool used = false;
    std::vector<int32_t> plane_cts; // CritTimeStep of each z plane
    std::vector<int64_t> active;    // substrate seeds (initially active cells), ascending; GrainID rank + 1
};

// A fully initialised problem, ready to be admitted to a device pool.
struct Problem {
    InputConfig cfg;
    Geometry g;
    // per-cell fields over the whole domain (index k*mx*my + i*my + j, y fastest); for a type-C
    // problem (dir.used) empty until materialize_fields fills them
    mutable std::vector<int32_t> cts;      // CritTimeStep
    mutable std::vector<int8_t> layer_id;  // LayerID (single layer: -1 or 0)
    mutable std::vector<float> du;         // UndercoolingChange
    mutable std::vector<int8_t> cell_type; // CellType
    mutable std::vector<int32_t> grain_id; // GrainID
    mutable std::vector<uint8_t> melted;   // Melted
    DirectionalSeeds dir;
    std::shared_ptr<std::mutex> fields_mutex = std::make_shared<std::mutex>();
    // orientation table: 9 floats per orientation (src/CAinitialize.cpp:1408-1441)
    std::vector<float> guv;
    // fresh-octahedron critical diagonal lengths, 26 per orientation
    std::vector<float> cdl_table;
    // potential nuclei in the reference's order (src/CAinitialize.cpp:2240-2247)
    std::vector<int32_t> nuclei_loc, nuclei_time;
    // interfacial response constants after the dt/dx normalisation of src/runCA.cpp:198-200
    double A_n = 0, B_n = 0, C_n = 0, D_n = 0;
    float du_value = 0.0f; // the one non-zero UndercoolingChange value of this problem (C and S; R with one value)
    // type R: the distinct non-zero UndercoolingChange values (ascending) when there are several, and
    // per cell the index of its value (0 for cells whose value is 0: their undercooling stays 0)
    std::vector<float> du_values;
    std::vector<uint16_t> du_class;
    // type R: per layer, the cycle at which the layer's temperature data ends (FinishTimeStep)
    std::vector<int> finish_time_step;
    int possible_nuclei = 0;
    double init_seconds = 0.0;
    // baseplate grain centres (x, y, z triples) for the device Voronoi pass of S problems
    std::vector<int32_t> voronoi_seeds;
    bool pinned = false;
};

// GrainID placeholder for substrate cells whose Voronoi assignment is computed on the device.
constexpr int32_t kVoronoiPending = INT32_MIN;

// Parses an ExaCA input file (and its material file); throws std::runtime_error with the
// reference's messages on malformed input. `log` receives the reference's rank-0 stdout lines.
void read_input_file(const std::string &path, InputConfig &cfg, std::string &log);

// Locates a data file the way checkFileInstalled does (src/CAinitialize.cpp:217-229): the
// install directory first, then the source data directory. Here: $EXACA_DATA_DIR, then the
// package's data directory.
std::string find_data_file(const std::string &name, const std::string &type, std::string &log);

// Builds the geometry, temperature field, substrate, grains and nuclei of a C or S problem
// (src/CAinitialize.cpp:579-2769). Throws for unsupported problem kinds.
void initialize_problem(Problem &p, std::string &log);

// Fills the per-cell host fields of a problem whose fields are made on the device (type C); a
// no-op when they are already there. Safe to call from several threads.
void materialize_fields(const Problem &p);

// Page-locks the per-cell host vectors (cudaHostRegister) for fast admission copies.
void pin_problem(Problem &p);
void unpin_problem(Problem &p);

// Host tables derived from the orientation file.
void read_orientations(const std::string &path, std::vector<float> &guv);
void build_cdl_table(const std::vector<float> &guv, std::vector<float> &table);

// Output writers (src/CAprint.cpp:170-571), byte-compatible with the reference. `threads` host
// threads format the z planes (<= 0: $EXACA_OUTPUT_THREADS, else every hardware thread); the
// bytes do not depend on it.
void write_vtk_fields(const Problem &p, const int32_t *grain_id, const std::string &fname, int threads = 0);
void write_misorientations(const Problem &p, const int32_t *grain_id, const std::string &fname,
                           std::string &log, int threads = 0);
void write_debug_vtk(const Problem &p, const std::string &fname);

struct RunTimes {
    double init = 0, run = 0, out = 0, nucl = 0, capture = 0, ghost = 0;
};
void write_log(const Problem &p, const std::string &fname, int cycle, const RunTimes &t, std::string &out);

// neighbour offsets in the reference's order (kNeighborX / Y / Z) are in directions.hpp
// ItList(9,26) and the per-case list lengths (src/CAinitialize.cpp:676-745)
void build_itlist(int itlist[9][26], int lens[9]);
inline int find_it_bounds(int rx, int ry, int mx, int my) {
    // src/CAfunctions.cpp:169-213
    if (ry == 0)
        return rx == 0 ? 5 : (rx == mx - 1 ? 6 : 1);
    if (ry == my - 1)
        return rx == 0 ? 7 : (rx == mx - 1 ? 8 : 2);
    return rx == 0 ? 3 : (rx == mx - 1 ? 4 : 0);
}

// Growth-increment table: entry n is the diagonal-length increment of an active cell whose
// undercooling is the n-fold float sum of du (src/CAupdate.cpp:236-261). Entry 0 is U = 0.
void build_growth_table(const Problem &p, float du, int n_entries, double *growth);
void build_growth_table(const Problem &p, int n_entries, std::vector<double> &growth);
// Most distinct UndercoolingChange values a problem may have (one growth table each).
constexpr int kMaxUndercoolingValues = 1024;

} // namespace exaca
