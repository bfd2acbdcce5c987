// ExaCA input-file parser for the B200 solver.
//
// Keeps the reference's file format exactly (src/CAinitialize.cpp:24-576): lines before a "*****"
// separator are skipped, then keys are read in a fixed order per problem type, a key matches when
// the expected text is a substring of the text before the colon, all whitespace is removed from
// the value, Y/N flags are strict, and the same runtime_error messages are raised.
#include "exaca_host.hpp"

#include <dlfcn.h>

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace exaca {

namespace {

struct LineReader {
    std::ifstream in;
    explicit LineReader(const std::string &path) : in(path) {}
    bool next(std::string &line) { return static_cast<bool>(std::getline(in, line)); }
};

// src/CAinitialize.cpp:24-30
void skip_to_separator(LineReader &r, const std::string &sep = "*****") {
    std::string line;
    while (r.next(line)) {
        if (line == sep)
            break;
    }
}

// src/CAinitialize.cpp:36-62. The deprecated-key loop only skips a line whose key contains every
// deprecated phrase; any other line ends the loop. That behaviour is kept as is.
std::string next_key(LineReader &r, std::string &line, std::size_t &colon) {
    static const char *deprecated[] = {"Burst buffer", "Source of input length unit"};
    bool again = true;
    std::string key;
    while (again) {
        line.clear();
        r.next(line);
        colon = line.find(':');
        key = line.substr(0, colon);
        if (colon == std::string::npos)
            throw std::runtime_error("Input \"" + key + "\" must be separated from value by \":\".");
        for (const char *d : deprecated) {
            if (key.find(d) != std::string::npos) {
                // warning printed by the reference; the flag is left as it was
            }
            else {
                again = false;
            }
        }
    }
    return key;
}

// src/CAinitialize.cpp:65-71: drop every whitespace character after the colon
std::string strip_value(const std::string &line, std::size_t colon) {
    std::string v = line.substr(colon + 1);
    std::string out;
    out.reserve(v.size());
    for (char c : v)
        if (!(c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v'))
            out.push_back(c);
    return out;
}

std::string parse_value(LineReader &r, const std::string &key) {
    std::string line;
    std::size_t colon;
    std::string k = next_key(r, line, colon);
    if (k.find(key) == std::string::npos)
        throw std::runtime_error("Required input not present: \"" + key + "\" not found in the input file");
    return strip_value(line, colon);
}

std::string parse_value_either(LineReader &r, const std::string &k1, const std::string &k2, int &which) {
    std::string line;
    std::size_t colon;
    std::string k = next_key(r, line, colon);
    if (k.find(k1) == std::string::npos) {
        if (k.find(k2) == std::string::npos)
            throw std::runtime_error("Required input not present: Neither " + k1 + " nor " + k2 +
                                     " was found in the input file");
        which = 2;
    }
    else {
        which = 1;
    }
    return strip_value(line, colon);
}

bool parse_flag(LineReader &r, const std::string &key) {
    std::string v = parse_value(r, key);
    if (v == "N")
        return false;
    if (v == "Y")
        return true;
    throw std::runtime_error("Input \"" + key + "\" must be \"Y\" or \"N\".");
}

bool file_opens(const std::string &path) {
    std::ifstream s(path);
    return s.is_open();
}

// src/CAinitialize.cpp:201-215
void require_file(const std::string &path, const std::string &type, std::string &log) {
    if (!file_opens(path))
        throw std::runtime_error("Could not locate/open " + type + " file");
    log += type + " file " + path + " opened\n";
}

int to_int(const std::string &v) { return std::stoi(v, nullptr, 10); }

std::string fmt(double v) {
    std::ostringstream s;
    s << v;
    return s.str();
}

// The package's data directory: <package>/data next to <package>/lib/libexaca_b200.so.
std::string package_data_dir() {
    Dl_info info;
    if (dladdr((void *)&package_data_dir, &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        std::size_t a = so.rfind('/');
        std::string lib = a == std::string::npos ? std::string(".") : so.substr(0, a);
        std::size_t b = lib.rfind('/');
        std::string pkg = b == std::string::npos ? std::string("..") : lib.substr(0, b);
        return pkg + "/data";
    }
    return "data";
}

} // namespace

std::string find_data_file(const std::string &name, const std::string &type, std::string &log) {
    const char *env = std::getenv("EXACA_DATA_DIR");
    if (env) {
        std::string f = std::string(env) + "/" + type + "/" + name;
        if (file_opens(f)) {
            log += type + " file " + f + " opened\n";
            return f;
        }
    }
    std::string f = package_data_dir() + "/" + type + "/" + name;
    require_file(f, type, log);
    return f;
}

void read_input_file(const std::string &path, InputConfig &c, std::string &log) {
    c.input_file = path;
    require_file(path, "Input", log);
    LineReader in(path);
    skip_to_separator(in);

    c.simulation_type = parse_value(in, "Problem type");
    c.decomposition_strategy = to_int(parse_value(in, "Decomposition strategy"));

    c.material_name = parse_value(in, "Material");
    std::string material_file = find_data_file(c.material_name, "Materials", log);
    {
        LineReader m(material_file);
        skip_to_separator(m);
        c.A = atof(parse_value(m, "A").c_str());
        c.B = atof(parse_value(m, "B").c_str());
        c.C = atof(parse_value(m, "C").c_str());
        c.D = atof(parse_value(m, "D").c_str());
        c.freezing_range = atof(parse_value(m, "Alloy freezing range").c_str());
    }

    c.deltax = atof(parse_value(in, "Cell size").c_str()) * pow(10, -6);
    c.nread = atof(parse_value(in, "Heterogeneous nucleation density").c_str());
    c.nmax = c.nread * pow(10, 12);
    c.dTN = atof(parse_value(in, "Mean nucleation undercooling").c_str());
    c.dTsigma = atof(parse_value(in, "Standard deviation of nucleation undercooling").c_str());
    c.path_to_output = parse_value(in, "Path to output");
    c.output_file = parse_value(in, "Output file base name");
    std::string orientation_name = parse_value(in, "File of grain orientations");
    c.orientation_file = find_data_file(orientation_name, "Substrate", log);

    const std::string &T = c.simulation_type;
    if (T == "R") {
        log += "CA Simulation using reduced temperature data from file(s)\n";
        c.ht_deltax = atof(parse_value(in, "Heat transport data mesh size").c_str()) * pow(10, -6);
        log += "Mesh size of the temperature data is " + fmt(c.ht_deltax) + " microns\n";
        std::string v = parse_value(in, "Time step");
        c.deltat = atof(v.c_str()) * pow(10, -6);
        log += "The time step is " + v + " microseconds\n";
        int which = 0;
        v = parse_value_either(in, "Path to substrate file", "Substrate grain spacing", which);
        if (which == 1) {
            c.substrate_file_name = v + "/" + parse_value(in, "Substrate file name");
            c.use_substrate_file = true;
            require_file(c.substrate_file_name, "Substrate", log);
        }
        else {
            c.substrate_grain_spacing = atof(v.c_str());
            c.use_substrate_file = false;
        }
        c.temppath = parse_value(in, "Path to temperature file");
        c.tempfile = parse_value(in, "Temperature filename");
        c.temp_files_in_series = to_int(parse_value(in, "Number of temperature files"));
        c.remelting = false;
        if (c.temp_files_in_series > 1)
            log += "Temperature data files are *" + c.tempfile + " , and there are " +
                   std::to_string(c.temp_files_in_series) + " in the series\n";
        else
            log += "The temperature data file is " + c.tempfile + "\n";
        for (int i = 1; i <= c.temp_files_in_series; i++) {
            std::string p = c.temppath + "/";
            p += c.temp_files_in_series > 1 ? std::to_string(i) + c.tempfile : c.tempfile;
            require_file(p, "Temperature", log);
        }
        c.extra_walls = parse_flag(in, "Extra set of wall cells around temperature field");
        c.number_of_layers = to_int(parse_value(in, "Number of layers"));
        c.layer_height = to_int(parse_value(in, "Offset between layers"));
        log += "A total of " + std::to_string(c.number_of_layers) + " of solidification offset by " +
               std::to_string(c.layer_height) + " CA cells will be simulated\n";
    }
    else if (T == "C") {
        c.number_of_layers = 1;
        c.layer_height = c.nz; // nz is still 0 here, as in the reference
        c.G = atof(parse_value(in, "Thermal gradient").c_str());
        c.R = atof(parse_value(in, "Cooling rate").c_str());
        log += "CA Simulation using a fixed thermal gradient of " + fmt(c.G) + " K/m and a cooling rate of " +
               fmt(c.R) + " K/s\n";
        c.nx = to_int(parse_value(in, "Domain size in x")) + 2;
        c.ny = to_int(parse_value(in, "Domain size in y")) + 2;
        c.nz = to_int(parse_value(in, "Domain size in z")) + 2;
        log += "The domain size is " + std::to_string(c.nx) + " by " + std::to_string(c.ny) + " by " +
               std::to_string(c.nz) + " cells\n";
        int nratio = to_int(parse_value(in, "\"N\""));
        c.deltat = c.deltax / (nratio * (c.R / c.G));
        log += "The time step is " + fmt(c.deltat * pow(10, 6)) + " microseconds\n";
        c.fract_surface_sites_active = atof(parse_value(in, "Fraction of surface sites active").c_str());
        log += "The fraction of CA cells at the bottom surface that are active is " +
               fmt(c.fract_surface_sites_active) + "\n";
    }
    else if (T == "S") {
        c.G = atof(parse_value(in, "Thermal gradient").c_str());
        c.R = atof(parse_value(in, "Cooling rate").c_str());
        log += "CA Simulation using a fixed thermal gradient of " + fmt(c.G) + " K/m and a cooling rate of " +
               fmt(c.R) + " K/s\n";
        c.nspots_x = to_int(parse_value(in, "Number of spots in x"));
        c.nspots_y = to_int(parse_value(in, "Number of spots in y"));
        float off = atof(parse_value(in, "Offset between spot centers").c_str());
        c.spot_offset = off * 1.0 * pow(10, -6) / c.deltax;
        float rad = atof(parse_value(in, "Radii of spots").c_str());
        c.spot_radius = rad * 1.0 * pow(10, -6) / c.deltax;
        c.number_of_layers = to_int(parse_value(in, "Number of layers"));
        c.layer_height = to_int(parse_value(in, "Offset between layers"));
        log += "A total of " + std::to_string(c.number_of_layers) +
               " spots per layer, with layers offset by " + std::to_string(c.layer_height) +
               " CA cells will be simulated\n";
        int nratio = to_int(parse_value(in, "\"N\""));
        c.deltat = c.deltax / (nratio * (c.R / c.G));
        log += "The time step is " + fmt(c.deltat * pow(10, 6)) + " microseconds\n";
        int which = 0;
        std::string v = parse_value_either(in, "Path to substrate file", "Substrate grain spacing", which);
        if (which == 1) {
            c.substrate_file_name = v + "/" + parse_value(in, "Substrate file name");
            c.use_substrate_file = true;
            require_file(c.substrate_file_name, "Substrate", log);
        }
        else {
            c.substrate_grain_spacing = atof(v.c_str());
            c.use_substrate_file = false;
        }
        c.nz = c.spot_radius + 3 + (c.number_of_layers - 1) * c.layer_height;
        c.nx = 4 + 2 * c.spot_radius + c.spot_offset * (c.nspots_x - 1);
        c.ny = 4 + 2 * c.spot_radius + c.spot_offset * (c.nspots_y - 1);
        log += "The domain size is " + std::to_string(c.nx) + " by " + std::to_string(c.ny) + " by " +
               std::to_string(c.nz) + " cells\n";
    }

    int which = 0;
    std::string v =
        parse_value_either(in, "Print file of grain orientations", "Output data printing options", which);
    if (which == 1) {
        log += "Warning: old input file format detected - code no longer supports some printing options. The "
               "code will still output Paraview vtk file of grain misorientations if that option is toggled in "
               "the input file; other toggled output data options will trigger the printing of a separate vtk "
               "file of layer ID, grain ID, and melting status of all cells. Obtaining data from this (such as "
               "grain area values, of grain orientation frequencies) are now done via post-processing rather "
               "than as part of ExaCA\n";
        bool old[6] = {false, false, false, false, false, false};
        c.print_debug = 0;
        if (v == "Y")
            old[0] = true;
        old[1] = parse_flag(in, "Print csv file of grain id values");
        old[2] = parse_flag(in, "Print csv file of ExaConstit-formatted grain id values");
        old[3] = parse_flag(in, "Print Paraview vtk file of grain misorientation values");
        old[4] = parse_flag(in, "Print file of grain area values");
        old[5] = parse_flag(in, "Print file of weighted grain area value");
        c.print_misorientation = old[3];
        c.print_full_output = (old[0] + old[1] + old[2] + old[4] + old[5]) > 0;
    }
    else if (which == 2) {
        c.print_misorientation = parse_flag(in, "Paraview vtk file of grain misorientation");
        c.print_full_output = parse_flag(in, "Paraview vtk file of all ExaCA data");
        bool dbg_a = parse_flag(in, "Print data for main Kokkos views");
        bool dbg_b = parse_flag(in, "Print data for all main data structures");
        c.print_debug = dbg_b ? 2 : (dbg_a ? 1 : 0);
    }

    log += "Decomposition Strategy is " + std::to_string(c.decomposition_strategy) + "\n";
    log += "Material simulated is " + c.material_name + ", interfacial response function constants are A = " +
           fmt(c.A) + ", B = " + fmt(c.B) + ", C = " + fmt(c.C) + ", and D = " + fmt(c.D) + "\n";
    log += "CA cell size is " + fmt(c.deltax * pow(10, 6)) + " microns\n";
    log += "Nucleation density is " + fmt(c.nread) + " x 10^12 per m^3\n";
    log += "Mean nucleation undercooling is " + fmt(c.dTN) + " K, standard deviation of distribution is " +
           fmt(c.dTsigma) + "K\n";
}

} // namespace exaca
