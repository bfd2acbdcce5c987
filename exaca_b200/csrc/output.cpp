// Output writers of the B200 solver: the ASCII legacy-VTK field file, the misorientation file, the
// init debug file and the run log. The byte layout is the reference's (src/CAprint.cpp:285-571):
// same headers, same (k, j, i) value order with x fastest, one line per z plane, every value
// followed by a space. Values are formatted with a buffered integer formatter instead of
// iostreams, which gives identical text for ints.
#include "exaca_host.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace exaca {

namespace {

class TextOut {
  public:
    explicit TextOut(const std::string &fname) : f_(std::fopen(fname.c_str(), "wb")) {
        if (!f_)
            throw std::runtime_error("could not open output file " + fname);
        buf_.resize(1 << 22);
    }
    ~TextOut() {
        flush();
        if (f_)
            std::fclose(f_);
    }
    void put(const std::string &s) {
        for (char c : s)
            putc_(c);
    }
    void put_int(long v) {
        char tmp[24];
        int n = 0;
        bool neg = v < 0;
        unsigned long u = neg ? (unsigned long)(-(v + 1)) + 1 : (unsigned long)v;
        do {
            tmp[n++] = (char)('0' + u % 10);
            u /= 10;
        } while (u);
        if (neg)
            putc_('-');
        while (n)
            putc_(tmp[--n]);
    }
    void put_fixed(float v) {
        char tmp[64];
        int n = std::snprintf(tmp, sizeof(tmp), "%f", (double)v);
        for (int i = 0; i < n; i++)
            putc_(tmp[i]);
    }
    void putc_(char c) {
        if (pos_ == buf_.size())
            flush();
        buf_[pos_++] = c;
    }
    void flush() {
        if (pos_ && f_)
            std::fwrite(buf_.data(), 1, pos_, f_);
        pos_ = 0;
    }

  private:
    std::FILE *f_;
    std::vector<char> buf_;
    size_t pos_ = 0;
};

// Whole-domain view of a rank-local field without the ghost ring: value at (k, x, y) for
// x in [0, nx), y in [0, ny); planes k = 0 and k = nz - 1 read as zero (src/CAprint.cpp:18-29,
// where the whole-domain arrays start zero-filled).
template <class T> long whole(const Geometry &g, const T *f, int k, int x, int y) {
    if (k == 0 || k == g.nz - 1)
        return 0;
    return (long)f[(long)k * g.mx * g.my + (long)(x + 1) * g.my + (y + 1)];
}

void vtk_header(TextOut &o, int nx, int ny, int nz) {
    o.put("# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET STRUCTURED_POINTS\n");
    o.put("DIMENSIONS " + std::to_string(nx) + " " + std::to_string(ny) + " " + std::to_string(nz) + "\n");
    o.put("ORIGIN 0 0 0\nSPACING 1 1 1\n");
    o.put("POINT_DATA " + std::to_string(nx * ny * nz) + "\n");
}

template <class T> void int_block(TextOut &o, const Geometry &g, const char *name, const T *f) {
    o.put(std::string("SCALARS ") + name + " int 1\nLOOKUP_TABLE default\n");
    for (int k = 0; k < g.nz; k++) {
        for (int j = 0; j < g.ny; j++)
            for (int i = 0; i < g.nx; i++) {
                o.put_int(whole(g, f, k, i, j));
                o.putc_(' ');
            }
        o.putc_('\n');
    }
}

void float_block(TextOut &o, const Geometry &g, const char *name, const float *f) {
    o.put(std::string("SCALARS ") + name + " float 1\nLOOKUP_TABLE default\n");
    for (int k = 0; k < g.nz; k++) {
        for (int j = 0; j < g.ny; j++)
            for (int i = 0; i < g.nx; i++) {
                float v = (k == 0 || k == g.nz - 1) ? 0.0f : f[(long)k * g.mx * g.my + (long)(i + 1) * g.my + (j + 1)];
                o.put_fixed(v);
                o.putc_(' ');
            }
        o.putc_('\n');
    }
}

} // namespace

void write_vtk_fields(const Problem &p, const int32_t *grain_id, const std::string &fname) {
    // src/CAprint.cpp:285-346 with PrintFullOutput: LayerID, GrainID, Melted
    TextOut o(fname);
    const Geometry &g = p.g;
    vtk_header(o, g.nx, g.ny, g.nz);
    int_block(o, g, "LayerID", p.layer_id.data());
    int_block(o, g, "GrainID", grain_id);
    int_block(o, g, "Melted", p.melted.data());
}

void write_debug_vtk(const Problem &p, const std::string &fname) {
    // src/CAprint.cpp:285-395 with PrintFullOutput false: the init debug dump of PrintDebug 1 or 2
    TextOut o(fname);
    const Geometry &g = p.g;
    vtk_header(o, g.nx, g.ny, g.nz);
    int_block(o, g, "LayerID", p.layer_id.data());
    if (p.cfg.print_debug == 2) {
        int_block(o, g, "GrainID", p.grain_id.data());
        int_block(o, g, "Melted", p.melted.data());
    }
    int_block(o, g, "CritTimeStep", p.cts.data());
    int_block(o, g, "CellType", p.cell_type.data());
    if (p.cfg.print_debug == 2) {
        float_block(o, g, "UndercoolingChange", p.du.data());
        std::vector<float> zeros(g.domain_size, 0.0f); // UndercoolingCurrent is 0 after init
        float_block(o, g, "Melted", zeros.data());
    }
}

void write_misorientations(const Problem &p, const int32_t *grain_id, const std::string &fname, std::string &log) {
    // src/CAprint.cpp:398-460
    const Geometry &g = p.g;
    TextOut o(fname);
    o.put("# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET STRUCTURED_POINTS\n");
    o.put("DIMENSIONS " + std::to_string(g.nx - 2) + " " + std::to_string(g.ny - 2) + " " +
          std::to_string(g.nz - 2) + "\n");
    o.put("ORIGIN 0 0 0\nSPACING 1 1 1\n");
    o.put("POINT_DATA " + std::to_string((g.nx - 2) * (g.ny - 2) * (g.nz - 2)) + "\n");
    o.put("SCALARS Angle_z int 1\nLOOKUP_TABLE default\n");
    std::vector<int> rounded(kNumOrientations);
    for (int n = 0; n < kNumOrientations; n++) {
        double amin = 62.7;
        for (int ll = 0; ll < 3; ll++) {
            double a = std::abs((180 / M_PI) * acos(p.guv[9 * n + 3 * ll + 2]));
            if (a < amin)
                amin = a;
        }
        rounded[n] = round(amin);
    }
    int nucleated = 0, melted = 0;
    for (int k = 1; k < g.nz - 1; k++) {
        for (int j = 1; j < g.ny - 1; j++)
            for (int i = 1; i < g.nx - 1; i++) {
                long idx = (long)k * g.mx * g.my + (long)(i + 1) * g.my + (j + 1);
                if (p.melted[idx] == 0) {
                    o.put("200 ");
                }
                else {
                    melted++;
                    int gid = grain_id[idx];
                    int ori = (std::abs(gid) - 1) % kNumOrientations;
                    if (ori < 0)
                        ori += kNumOrientations;
                    int angle;
                    if (gid < 0) {
                        angle = rounded[ori] + 100;
                        nucleated++;
                    }
                    else {
                        angle = rounded[ori];
                    }
                    o.put_int(angle);
                    o.putc_(' ');
                }
            }
        o.putc_('\n');
    }
    std::ostringstream s;
    s << "Volume fraction of solidified portion of domain claimed by nucleated grains: "
      << (float)(nucleated) / (float)(melted) << "\n";
    log += s.str();
}

void write_log(const Problem &p, const std::string &fname, int cycle, const RunTimes &t, std::string &out) {
    // src/CAprint.cpp:463-571 (one rank)
    const InputConfig &c = p.cfg;
    const Geometry &g = p.g;
    std::ostringstream L;
    double total = t.init + t.run + t.out;
    L << "log file for a simulation run with input file " << c.input_file << "  run on " << 1
      << " MPI ranks, output written at cycle " << cycle << "\n";
    L << "This simulation took " << total << " seconds to run, with the init/run/output breakdown as " << t.init
      << "/" << t.run << "/" << t.out << "\n";
    L << "This simulation was type: " << c.simulation_type << "\n";
    L << "Domain size in x: " << g.nx << "\n";
    L << "Domain size in y: " << g.ny << "\n";
    L << "Domain size in z: " << g.nz << "\n";
    L << "Cell size: " << c.deltax << " microns" << "\n";
    L << "Time step: " << c.deltat << " microseconds" << "\n";
    L << "Nucleation density was " << c.nmax << " m^-3 , mean nucleation undercooling was " << c.dTN
      << " K, and standard deviation of nucleation undercooling was " << c.dTsigma << " K" << "\n";
    L << "Interfacial response function parameters used were " << p.A_n << " , " << p.B_n << " , " << p.C_n
      << " , " << p.D_n << " , and the alloy freezing range was " << c.freezing_range << "\n";
    if (c.simulation_type == "C") {
        L << "The thermal gradient was " << c.G << " K/m, and the cooling rate " << c.R << " K/s" << "\n";
        L << "The fraction of surface sites active was " << c.fract_surface_sites_active << "\n";
    }
    else if (c.simulation_type == "S") {
        L << "A total of " << c.nspots_x << " in X and " << c.nspots_y << " in Y were considered" << "\n";
        L << "The spots were offset by " << c.spot_offset << " microns, and had radii of " << c.spot_radius
          << " microns" << "\n";
        L << "This pattern was repeated for " << c.number_of_layers << " layers" << "\n";
    }
    L << "The decomposition scheme used was: " << c.decomposition_strategy << "\n";
    L << "Rank " << 0 << " contained " << g.mx << " cells in x , " << g.my << " cells in y; subdomain was offset by "
      << g.xoff << " in x , " << g.yoff << " in y" << "\n";
    L << "Max/min rank time initializing data  = " << t.init << " / " << t.init << " s" << "\n";
    L << "Max/min rank time in CA nucleation   = " << t.nucl << " / " << t.nucl << " s" << "\n";
    L << "Max/min rank time in CA cell capture = " << t.capture << " / " << t.capture << " s" << "\n";
    L << "Max/min rank time in CA ghosting     = " << t.ghost << " / " << t.ghost << " s" << "\n";
    L << "Max/min rank time exporting data     = " << t.out << " / " << t.out << " s\n" << "\n";
    std::ofstream f(fname, std::ios::binary);
    if (!f)
        throw std::runtime_error("could not open log file " + fname);
    f << L.str();

    std::ostringstream O;
    O << "===================================================================================\n";
    O << "Having run with = 1 processors\n";
    O << "Output written at cycle = " << cycle << "\n";
    O << "Total time = " << total << "\n";
    O << "Time spent initializing data = " << t.init << " s\n";
    O << "Time spent performing CA calculations = " << t.run << " s\n";
    O << "Time spent collecting and printing output data = " << t.out << " s\n\n";
    O << "Max/min rank time initializing data  = " << t.init << " / " << t.init << " s\n";
    O << "Max/min rank time in CA nucleation   = " << t.nucl << " / " << t.nucl << " s\n";
    O << "Max/min rank time in CA cell capture = " << t.capture << " / " << t.capture << " s\n";
    O << "Max/min rank time in CA ghosting     = " << t.ghost << " / " << t.ghost << " s\n";
    O << "Max/min rank time exporting data     = " << t.out << " / " << t.out << " s\n\n";
    O << "===================================================================================\n";
    out += O.str();
}

} // namespace exaca
