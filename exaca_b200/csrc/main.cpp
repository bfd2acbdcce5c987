// ExaCA-B200 executable: the drop-in for `ExaCA-Kokkos <input file>` (src/main.cpp:15-47) at one
// rank. An optional second argument selects the CUDA device.
#include <cstdio>
#include <cstdlib>

#include "../../include/exaca_b200.h"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "Error: Must provide path to input file on the command line.\n");
        return 1;
    }
    int device = argc > 2 ? std::atoi(argv[2]) : 0;
    int rc = exaca_run_program(argv[1], device);
    if (rc != 0) {
        std::fprintf(stderr, "ExaCA-B200 error %d: %s\n", rc, exaca_last_error());
        return 1;
    }
    return 0;
}
