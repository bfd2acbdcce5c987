// Output writers of the B200 solver: the ASCII legacy-VTK field file, the misorientation file, the
// init debug file and the run log. The byte layout is the reference's (src/CAprint.cpp:285-571):
// same headers, same (k, j, i) value order with x fastest, one line per z plane, every value
// followed by a space. Values are formatted with an integer digit loop instead of iostreams (the
// same text for ints), one z plane per task on all host threads, and written in plane order.
#include "exaca_host.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <thread>

namespace exaca {

namespace {

// Text of one z plane, built with plain appends (ints by a digit loop; floats by "%f", which is
// what `std::fixed` iostream output prints). One cache line each: threads append to neighbouring
// planes at the same time.
class alignas(64) PlaneText {
  public:
    void clear() { n_ = 0; }
    void reserve(size_t bytes) {
        if (buf_.size() < bytes)
            buf_.resize(bytes);
    }
    void put(const char *s, size_t len) {
        need(len);
        std::memcpy(buf_.data() + n_, s, len);
        n_ += len;
    }
    void put_int(long v) {
        need(24);
        char tmp[24];
        int n = 0;
        bool neg = v < 0;
        unsigned long u = neg ? (unsigned long)(-(v + 1)) + 1 : (unsigned long)v;
        do {
            tmp[n++] = (char)('0' + u % 10);
            u /= 10;
        } while (u);
        if (neg)
            buf_[n_++] = '-';
        while (n)
            buf_[n_++] = tmp[--n];
    }
    void put_fixed(float v) {
        need(64);
        n_ += (size_t)std::snprintf(buf_.data() + n_, 64, "%f", (double)v);
    }
    void putc_(char c) {
        need(1);
        buf_[n_++] = c;
    }
    const char *data() const { return buf_.data(); }
    size_t size() const { return n_; }

  private:
    void need(size_t len) {
        if (n_ + len > buf_.size())
            buf_.resize(std::max(buf_.size() * 2, n_ + len + 4096));
    }
    std::vector<char> buf_;
    size_t n_ = 0;
};

class File {
  public:
    explicit File(const std::string &fname) : f_(std::fopen(fname.c_str(), "wb")) {
        if (!f_)
            throw std::runtime_error("could not open output file " + fname);
    }
    ~File() {
        if (f_)
            std::fclose(f_);
    }
    void put(const std::string &s) { write(s.data(), s.size()); }
    void write(const char *p, size_t n) {
        if (n && std::fwrite(p, 1, n, f_) != n)
            throw std::runtime_error("write to output file failed");
    }

  private:
    std::FILE *f_;
};

int output_threads() {
    if (const char *e = std::getenv("EXACA_OUTPUT_THREADS")) {
        int t = std::atoi(e);
        if (t > 0)
            return t;
    }
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

// Formats planes 0..n-1 with `plane(k, text)` on `threads` host threads, a batch of planes at a
// time (bounded memory), and writes them to `f` in plane order; the writes of one batch overlap
// the formatting of the next. The bytes are those of formatting the planes one after another.
template <class Fn> void write_planes(File &f, int n, int threads, size_t plane_bytes, Fn &&plane) {
    threads = std::max(1, std::min(threads, n));
    const int batch = threads * 4;
    std::vector<PlaneText> sets[2] = {std::vector<PlaneText>(batch), std::vector<PlaneText>(batch)};
    std::thread writer;
    std::exception_ptr werr;
    int s = 0;
    for (int b = 0; b < n; b += batch) {
        const int m = std::min(batch, n - b);
        std::vector<PlaneText> &set = sets[s];
        std::atomic<int> next{0};
        std::exception_ptr ferr;
        std::mutex ferr_mu;
        auto work = [&] {
            try {
                for (int i; (i = next.fetch_add(1)) < m;) {
                    set[i].clear();
                    set[i].reserve(plane_bytes);
                    plane(b + i, set[i]);
                }
            } catch (...) {
                std::lock_guard<std::mutex> lk(ferr_mu);
                ferr = std::current_exception();
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < std::min(threads, m); t++)
            pool.emplace_back(work);
        work();
        for (auto &t : pool)
            t.join();
        if (writer.joinable())
            writer.join();
        if (ferr)
            std::rethrow_exception(ferr);
        if (werr)
            std::rethrow_exception(werr);
        std::vector<PlaneText> *done = &set;
        writer = std::thread([&f, done, m, &werr] {
            try {
                for (int i = 0; i < m; i++)
                    f.write((*done)[i].data(), (*done)[i].size());
            } catch (...) {
                werr = std::current_exception();
            }
        });
        s ^= 1;
    }
    if (writer.joinable())
        writer.join();
    if (werr)
        std::rethrow_exception(werr);
}

// Whole-domain view of a rank-local field without the ghost ring: value at (k, x, y) for
// x in [0, nx), y in [0, ny); planes k = 0 and k = nz - 1 read as zero (src/CAprint.cpp:18-29,
// where the whole-domain arrays start zero-filled).
template <class T> long whole(const Geometry &g, const T *f, int k, int x, int y) {
    if (k == 0 || k == g.nz - 1)
        return 0;
    return (long)f[(long)k * g.mx * g.my + (long)(x + 1) * g.my + (y + 1)];
}

void vtk_header(File &o, int nx, int ny, int nz) {
    o.put("# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET STRUCTURED_POINTS\n");
    o.put("DIMENSIONS " + std::to_string(nx) + " " + std::to_string(ny) + " " + std::to_string(nz) + "\n");
    o.put("ORIGIN 0 0 0\nSPACING 1 1 1\n");
    o.put("POINT_DATA " + std::to_string((long)nx * ny * nz) + "\n");
}

template <class T> void int_block(File &o, const Geometry &g, const char *name, const T *f, int threads) {
    o.put(std::string("SCALARS ") + name + " int 1\nLOOKUP_TABLE default\n");
    write_planes(o, g.nz, threads, (size_t)g.nx * g.ny * 4 + 64, [&](int k, PlaneText &t) {
        for (int j = 0; j < g.ny; j++)
            for (int i = 0; i < g.nx; i++) {
                t.put_int(whole(g, f, k, i, j));
                t.putc_(' ');
            }
        t.putc_('\n');
    });
}

void float_block(File &o, const Geometry &g, const char *name, const float *f, int threads) {
    o.put(std::string("SCALARS ") + name + " float 1\nLOOKUP_TABLE default\n");
    write_planes(o, g.nz, threads, (size_t)g.nx * g.ny * 10 + 64, [&](int k, PlaneText &t) {
        for (int j = 0; j < g.ny; j++)
            for (int i = 0; i < g.nx; i++) {
                float v = (k == 0 || k == g.nz - 1) ? 0.0f : f[(long)k * g.mx * g.my + (long)(i + 1) * g.my + (j + 1)];
                t.put_fixed(v);
                t.putc_(' ');
            }
        t.putc_('\n');
    });
}

} // namespace

void write_vtk_fields(const Problem &p, const int32_t *grain_id, const std::string &fname, int threads) {
    // src/CAprint.cpp:285-346 with PrintFullOutput: LayerID, GrainID, Melted
    if (threads <= 0)
        threads = output_threads();
    materialize_fields(p);
    File o(fname);
    const Geometry &g = p.g;
    vtk_header(o, g.nx, g.ny, g.nz);
    int_block(o, g, "LayerID", p.layer_id.data(), threads);
    int_block(o, g, "GrainID", grain_id, threads);
    int_block(o, g, "Melted", p.melted.data(), threads);
}

void write_debug_vtk(const Problem &p, const std::string &fname) {
    // src/CAprint.cpp:285-395 with PrintFullOutput false: the init debug dump of PrintDebug 1 or 2
    const int threads = output_threads();
    materialize_fields(p);
    File o(fname);
    const Geometry &g = p.g;
    vtk_header(o, g.nx, g.ny, g.nz);
    int_block(o, g, "LayerID", p.layer_id.data(), threads);
    if (p.cfg.print_debug == 2) {
        int_block(o, g, "GrainID", p.grain_id.data(), threads);
        int_block(o, g, "Melted", p.melted.data(), threads);
    }
    int_block(o, g, "CritTimeStep", p.cts.data(), threads);
    int_block(o, g, "CellType", p.cell_type.data(), threads);
    if (p.cfg.print_debug == 2) {
        float_block(o, g, "UndercoolingChange", p.du.data(), threads);
        std::vector<float> zeros(g.domain_size, 0.0f); // UndercoolingCurrent is 0 after init
        float_block(o, g, "Melted", zeros.data(), threads);
    }
}

void write_misorientations(const Problem &p, const int32_t *grain_id, const std::string &fname, std::string &log,
                           int threads) {
    // src/CAprint.cpp:398-460
    if (threads <= 0)
        threads = output_threads();
    materialize_fields(p);
    const Geometry &g = p.g;
    File o(fname);
    o.put("# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET STRUCTURED_POINTS\n");
    o.put("DIMENSIONS " + std::to_string(g.nx - 2) + " " + std::to_string(g.ny - 2) + " " +
          std::to_string(g.nz - 2) + "\n");
    o.put("ORIGIN 0 0 0\nSPACING 1 1 1\n");
    o.put("POINT_DATA " + std::to_string((long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2)) + "\n");
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
    // per-plane counts, summed afterwards (the order of integer sums does not matter)
    std::vector<long> nucleated(g.nz, 0), melted(g.nz, 0);
    write_planes(o, g.nz - 2, threads, (size_t)g.nx * g.ny * 4 + 64, [&](int kk, PlaneText &t) {
        const int k = kk + 1;
        long nuc = 0, mel = 0;
        for (int j = 1; j < g.ny - 1; j++)
            for (int i = 1; i < g.nx - 1; i++) {
                long idx = (long)k * g.mx * g.my + (long)(i + 1) * g.my + (j + 1);
                if (p.melted[idx] == 0) {
                    t.put("200 ", 4);
                }
                else {
                    mel++;
                    int gid = grain_id[idx];
                    int ori = (std::abs(gid) - 1) % kNumOrientations;
                    if (ori < 0)
                        ori += kNumOrientations;
                    int angle;
                    if (gid < 0) {
                        angle = rounded[ori] + 100;
                        nuc++;
                    }
                    else {
                        angle = rounded[ori];
                    }
                    t.put_int(angle);
                    t.putc_(' ');
                }
            }
        t.putc_('\n');
        nucleated[k] = nuc;
        melted[k] = mel;
    });
    long n_nuc = 0, n_mel = 0;
    for (int k = 0; k < g.nz; k++) {
        n_nuc += nucleated[k];
        n_mel += melted[k];
    }
    // the reference counts in int and divides as float
    std::ostringstream s;
    s << "Volume fraction of solidified portion of domain claimed by nucleated grains: "
      << (float)((int)n_nuc) / (float)((int)n_mel) << "\n";
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
    else {
        L << c.number_of_layers << " layers were simulated, with an offset of " << c.layer_height << " cells" << "\n";
        L << (c.remelting ? "Remelting was included" : "Remelting was not included") << "\n";
        if (c.use_substrate_file)
            L << "The substrate file was " << c.substrate_file_name << "\n";
        else
            L << "The mean substrate grain size was " << c.substrate_grain_spacing << " microns" << "\n";
        if (c.simulation_type == "R") {
            L << "The " << c.temp_files_in_series << " temperature file(s) used had the name " << c.tempfile << "\n";
            L << "The temperature data resolution was " << c.ht_deltax << " microns" << "\n";
        }
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
