/*
 * C ABI of the B200-native ExaCA cellular-automaton solver (libexaca_b200.so).
 *
 * The reference (ExaCA, Kokkos + MPI) exposes no plugin or FFI layer: its boundary is the
 * ExaCA-Kokkos executable, the driver RunProgram_Reduced and the three step functions. Every entry
 * point below names the reference interface it replaces. All functions return 0 on success and a
 * negative error code otherwise (never throw across the ABI); exaca_last_error() returns the
 * message of the last failure on the calling thread. Pointers are plain host pointers; the library
 * owns all device memory. One pool is driven by one host thread at a time; separate pools may be
 * used from separate threads.
 */
#ifndef EXACA_B200_H
#define EXACA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EXACA_OK 0
#define EXACA_ERR_INPUT (-1)     /* malformed input file, missing key or data file */
#define EXACA_ERR_UNSUPPORTED (-2) /* a problem this solver does not handle (substrate file, >127 layers, ...) */
#define EXACA_ERR_CUDA (-3)      /* CUDA runtime failure or device-side error flag */
#define EXACA_ERR_BUDGET (-4)    /* admission refused: HBM budget or slot limit */
#define EXACA_ERR_ARG (-5)       /* bad handle, slot or size */

typedef struct exaca_problem exaca_problem; /* parsed and initialised host-side problem */
typedef struct exaca_pool exaca_pool;       /* device pool of domains */

/* Geometry of a problem (src/CAfunctions.cpp:34-166 at one rank). */
typedef struct {
    int nx, ny, nz;        /* global sizes including the wall layers */
    int mx, my;            /* MyXSlices, MyYSlices (nx + 2, ny + 2) */
    int nz_active;         /* active window height */
    int64_t domain_size;   /* mx * my * nz cells, index k*mx*my + i*my + j */
    int64_t active_size;   /* mx * my * nz_active */
    int n_nuclei;          /* potential nucleation sites */
    double deltat;         /* s */
    char simulation_type;  /* 'C' or 'S' */
} exaca_problem_geometry;

/* Parameters of a synthetic directional-solidification problem, equal to an input file of
 * problem type C with these values (keys of src/CAinitialize.cpp:395-441). */
typedef struct {
    int nx, ny, nz;                  /* "Domain size in x/y/z" (cells, without walls) */
    double cell_size_um;             /* "Cell size" */
    double G, R;                     /* "Thermal gradient" K/m, "Cooling rate" K/s */
    int n_ratio;                     /* "N": deltat = deltax / (N * R / G) */
    double nucleation_density;       /* "Heterogeneous nucleation density" (x 1e12 m^-3) */
    double dTN, dTsigma;             /* mean / sigma of the nucleation undercooling (K) */
    double fract_surface_active;     /* "Fraction of surface sites active" */
    double A, B, C, D, freezing_range; /* material file values */
} exaca_dirs_params;

/* Dynamic state of one pool slot. */
typedef struct {
    int cycle;          /* last executed CA cycle */
    int done;           /* 1 once the domain met the reference's termination test */
    int nn;             /* nucleation events so far */
    int error;          /* device error flags (0 = none; EXACA_FLAG_*) */
    int64_t liquid;     /* liquid cells left (device-checked single-layer slots) */
    int layer;          /* current layer (layernumber, src/runCA.cpp:282) */
    int window_z_lo;    /* the layer's active window: z planes [window_z_lo, window_z_lo + window_nz) */
    int window_nz;      /* (ZBound_Low and nzActive, src/runCA.cpp:96-102) */
    int reserved;
} exaca_domain_status;

/* Work counters of a pool since its creation (summed over all domains). */
typedef struct {
    uint64_t cycles;    /* CA cycles launched */
    uint64_t launches;  /* kernels launched by exaca_pool_step / run_plain / profile */
    uint64_t listed;    /* active-list entries visited */
    uint64_t grown;     /* active cells grown (eligible: cycle > CritTimeStep) */
    uint64_t captured;  /* liquid cells captured */
    uint64_t nucleated; /* nucleation events */
    uint64_t claims;    /* capture claims issued */
    uint64_t row_reads; /* critical-diagonal-length rows read (diagonal reached the cached minimum) */
    uint64_t dropped;   /* active-cell records dropped (solidified, or their domain finished) */
    uint64_t fresh;     /* liquid-neighbour masks built from the 26 neighbour types */
    uint64_t rechecks;  /* solidification re-checks next to claimed cells */
    uint64_t flagged;   /* records handed from the growth pass to the claim pass */
    uint64_t h2d_bytes; /* problem data copied host->device: cell fields (or, for type C, the seeds
                           they are made from on the device), nuclei, growth and orientation tables */
    uint64_t d2h_bytes; /* results copied device->host (GrainID, CellType, octahedron state) */
} exaca_pool_stats_t;

/* The reference's every-1000-cycle census (src/CAupdate.cpp:738-808). */
typedef struct {
    uint64_t superheated, undercooled, active, solid, remaining, next_cts;
} exaca_census;

const char *exaca_last_error(void);

/* Drop-in for RunProgram_Reduced(int id, int np, std::string InputFile) (src/runCA.hpp:11) and the
 * ExaCA-Kokkos main (src/main.cpp:15-47) at np = 1: reads the input file, initialises, solves on
 * CUDA device `device`, writes the .vtk / _Misorientations.vtk / .log outputs and prints the
 * reference's progress lines to stdout. */
int exaca_run_program(const char *input_file, int device);

/* Input parsing and initialisation: InputReadFromFile + ParallelMeshInit + TempInit_* +
 * OrientationInit + SubstrateInit_* + ActiveCellWallInit + GrainInit + NucleiInit
 * (src/CAinitialize.hpp:16-96; src/runCA.cpp:38-195). Host only; no device needed. */
int exaca_problem_from_file(const char *input_file, exaca_problem **out);
int exaca_problem_directional(const exaca_dirs_params *prm, exaca_problem **out);
void exaca_problem_free(exaca_problem *p);
int exaca_problem_info(const exaca_problem *p, exaca_problem_geometry *info);
/* Initial fields (domain_size values each; any pointer may be NULL). GrainID entries of
 * Voronoi-baseplate cells read INT32_MIN here; the device fills them in at admission. */
int exaca_problem_fields(const exaca_problem *p, int32_t *cell_type, int32_t *grain_id, int32_t *crit_time_step,
                         float *undercooling_change, int32_t *layer_id);
/* Page-locks the problem's host fields so that admission copies run at full PCIe bandwidth. */
int exaca_problem_pin(exaca_problem *p);
/* Bytes of HBM a problem takes in a pool slot. */
int64_t exaca_problem_slot_bytes(const exaca_problem *p);

/* Device pool: replaces the device-side views of src/runCA.cpp:232-256. budget_bytes bounds the
 * per-slot allocations (admission control); list_capacity sizes the shared active-cell list. */
int exaca_pool_create(int device, size_t budget_bytes, uint64_t list_capacity, exaca_pool **out);
void exaca_pool_destroy(exaca_pool *pool);
/* Uploads a problem (the host->device mirror copies of src/runCA.cpp:234-250) and finishes its
 * initialisation on the device. device_check = 1 lets the device end the domain at the
 * reference's termination test (at the 1000-cycle check that finds no liquid; once no liquid is
 * left, every cell is past its CritTimeStep and at least one more cycle has run, the domain ends
 * early with that check's cycle and the same fields); 0 leaves it to exaca_pool_run_plain. */
int exaca_pool_admit(exaca_pool *pool, const exaca_problem *p, int device_check, int *slot);
/* Advances every unfinished domain by n_cycles CA cycles: Nucleation + CellCapture
 * (src/CAupdate.hpp:15-29) per cycle, in one persistent kernel launch. Asynchronous. */
int exaca_pool_step(exaca_pool *pool, int n_cycles);
/* Batched solve (no counterpart in the reference): steps every admitted domain in chunks of
 * chunk_cycles until each has met the reference's termination test on the device (all slots must
 * be admitted with device_check = 1; type-C problems, whose run has no cycle jump). A domain's
 * result does not depend on the other domains in the pool. */
int exaca_pool_run_all(exaca_pool *pool, int chunk_cycles, int64_t max_cycles, int64_t *cycles_stepped);
/* Step configurations (no counterpart in the reference): config = mode * 4 + shape, mode 0 the
 * persistent kernel and 1 a CUDA graph of the per-pass kernels, shape one of the compiled
 * {capture lanes 4|8} x {growth records per lane 2|4}. Results do not depend on the configuration.
 * A configuration set here or chosen by exaca_pool_autotune stays; without either,
 * exaca_pool_run_plain picks the fastest persistent one itself. */
#define EXACA_STEP_CONFIGS 8
int exaca_pool_set_config(exaca_pool *pool, int config);
/* Grid of the persistent kernel (no counterpart in the reference): divisor d in 1-32 runs 1/d of
 * the co-resident blocks (cheaper grid-wide meetings for short active lists), 0 (the default) lets
 * the pool choose (exaca_pool_run_plain's trials, else the active list's length at the last status
 * read). Results do not depend on it. */
int exaca_pool_set_grid(exaca_pool *pool, int divisor);
/* Autotuner: runs trial_cycles real cycles of the pool's domains in every configuration, keeps the
 * fastest; ms_per_cycle (EXACA_STEP_CONFIGS entries, may be NULL) receives the trial times. */
int exaca_pool_autotune(exaca_pool *pool, int trial_cycles, int *config, double *ms_per_cycle);
/* exaca_pool_step with CUDA events around the launch: waits and returns its device time in ms. */
int exaca_pool_timed_step(exaca_pool *pool, int n_cycles, double *ms);
/* exaca_pool_step with the persistent kernel's device timeline on (globaltimer at every grid-wide
 * meeting point); waits and returns per-cycle averages in microseconds: us[7] = {growth pass done in
 * the first block, in the last block; claim pass first, last; capture pass first, last; end of the
 * cycle and start of the next (run by the last block alone)}. Pass times count from the release of
 * the previous meeting point. */
int exaca_pool_profile_persistent(exaca_pool *pool, int n_cycles, double *us);
/* Device error flags, as exaca_domain_status.error reports them. */
#define EXACA_FLAG_GROWTH_TABLE 1  /* undercooling count beyond the growth table */
#define EXACA_FLAG_LIST_OVERFLOW 2 /* active list or claim queue full */
#define EXACA_FLAG_BOUNDS 4        /* an index out of range */
#define EXACA_FLAG_BARRIER 8       /* a grid-wide wait of the persistent kernel gave up after 1 s */
/* Diagnostic, no counterpart in the reference: the persistent kernel's grid-wide wait run where
 * nothing can release it (two blocks, one of which leaves without arriving). The wait ends by its
 * 1 s limit; *flags receives the flags it left (EXACA_FLAG_BARRIER), which are then cleared, and
 * the pool stays usable. */
int exaca_pool_check_bounded_wait(exaca_pool *pool, int *flags);
/* Waits for the device and reads one slot's state. */
int exaca_pool_status(exaca_pool *pool, int slot, exaca_domain_status *st);
/* exaca_pool_status for n_slots slots with one device read (request loops poll many domains). */
int exaca_pool_status_many(exaca_pool *pool, int n_slots, const int *slots, exaca_domain_status *st);
/* Waits for the device and reads the pool's work counters (summed over all domains). */
int exaca_pool_stats(exaca_pool *pool, exaca_pool_stats_t *st);
/* IntermediateOutputAndCheck's census (src/CAupdate.hpp:30-33) for one slot. */
int exaca_pool_census(exaca_pool *pool, int slot, exaca_census *c);
/* Runs one slot to completion exactly as the reference's layer loop (src/runCA.cpp:290-342):
 * 1000-cycle census, termination, type-S cycle jump; progress lines are appended to stdout when
 * verbose is 1. Unless a step configuration was set, it times the four persistent ones (with all
 * and with half of the co-resident blocks, for active lists below 2^19 records) for 50 real cycles
 * each at cycle 1000 of a layer and every 4000 cycles after, and keeps the fastest; before the first
 * trials it runs all co-resident blocks. (exaca_pool_step and exaca_pool_run_all run a sixteenth of
 * them while the active list read at the last status holds fewer than 2^13 records.) */
int exaca_pool_run_plain(exaca_pool *pool, int slot, int verbose, int *final_cycle);
/* Ends the current layer of a multilayer slot and sets up the next: DomainShiftAndResize (the new
 * window from one plane below the lowest active cell to the highest cell of the next layer) and
 * LayerSetup (window octahedra cleared, fresh octahedra for its active cells), as the reference's
 * layer loop does between layers (src/runCA.cpp:344-390; src/CAinitialize.cpp:2772-2982); the
 * cycle restarts at 0. The reference's lines are appended to stdout when verbose is 1.
 * EXACA_ERR_ARG if the slot is in its last layer. */
int exaca_pool_next_layer(exaca_pool *pool, int slot, int verbose);
/* CUDA-event device time (ms) of the last exaca_pool_run_plain on this pool. */
double exaca_pool_last_run_ms(exaca_pool *pool);
/* Runs n_cycles cycles pass by pass as separate kernels with CUDA events around each launch and
 * returns the summed times in kernel_ms[4] = {cycle start + nucleation, growth pass, claim pass,
 * capture + neighbour re-check pass}. */
int exaca_pool_profile_cycles(exaca_pool *pool, int n_cycles, double *kernel_ms);
/* Device->host copy of GrainID and CellType (src/runCA.cpp:423-424); NULL skips a field. Page-locked
 * buffers take one DMA per field; pageable ones go through the pool's pinned staging pieces. */
int exaca_pool_copy_out(exaca_pool *pool, int slot, int32_t *grain_id, int32_t *cell_type);
/* exaca_pool_copy_out for a slot whose domain has ended as of the last exaca_pool_status(_many) /
 * run_plain: the copies use the pool's separate copy stream and do not wait for cycles launched
 * since, so a request loop can fetch finished results while the next cycles run (the reference's
 * copy-back, src/runCA.cpp:423-424, once per finished request). Returns when the data is on the
 * host; EXACA_ERR_ARG if the domain has not ended. */
int exaca_pool_copy_out_concurrent(exaca_pool *pool, int slot, int32_t *grain_id, int32_t *cell_type);
/* Active-window octahedron state (DiagonalLength, DOCenter x3, CritDiagonalLength x26) of the
 * slot's current layer: window_nz * mx * my cells from plane window_z_lo (exaca_pool_status), the
 * reference's window arrays (src/runCA.cpp:147-151, resized per layer at :352-356). */
int exaca_pool_copy_octahedra(exaca_pool *pool, int slot, float *dl, float *doc, float *cdl);
/* Frees a slot's device memory. */
int exaca_pool_retire(exaca_pool *pool, int slot);
int64_t exaca_pool_bytes_in_use(exaca_pool *pool);

/* Grain statistics of the reference analysis (analysis/src/GAprint.cpp:17-198: PrintMisorientationData,
 * PrintSizeData) computed on the device from a slot's GrainID field, without writing .vtk files. */
#define EXACA_MISORIENTATION_BINS 64
typedef struct {
    int64_t region_cells;               /* cells in the region */
    int64_t melted_cells;               /* region cells that melted */
    int64_t n_grains;                   /* distinct GrainIDs in the region */
    double mean_grain_volume_um3;       /* the reference's expression: deltax^2 * 1e12 * cells / grains */
    double nucleated_fraction;          /* region cells with a nucleated (negative) GrainID */
    double mean_misorientation_deg;     /* mean over melted cells of the grain's smallest angle to +Z */
    double mean_misorientation_top_deg; /* the same over the region's top plane */
    uint64_t misorientation_hist[EXACA_MISORIENTATION_BINS]; /* melted cells per 1-degree bin (last: >= 63) */
} exaca_grain_stats;
/* region: {xmin, xmax, ymin, ymax, zmin, zmax} in the coordinates of the .vtk output (whole domain
 * with walls, no ghost ring), or NULL for the interior without the wall layers. */
int exaca_pool_grain_stats(exaca_pool *pool, int slot, const int32_t *region, exaca_grain_stats *out);

/* Writes the reference's output files for a finished slot (src/CAprint.cpp:170-571). */
int exaca_pool_write_outputs(exaca_pool *pool, int slot, const exaca_problem *p, const char *path_prefix);

/* The .vtk / _Misorientations.vtk files that the problem's print flags ask for
 * (src/CAprint.cpp:170-460), from a host GrainID in the layout of
 * exaca_pool_copy_out, without a device. The z planes are formatted on `threads` host threads
 * (<= 0: $EXACA_OUTPUT_THREADS, else every hardware thread) and written in order; the bytes are
 * the reference's whatever the thread count. Replaces the rank-0 collect-and-print of
 * PrintExaCAData (src/CAprint.cpp:170-282): PrintCAFields (:285-395) and
 * PrintGrainMisorientations (:398-460). */
int exaca_problem_write_outputs(const exaca_problem *p, const int32_t *grain_id, const char *path_prefix,
                                int threads);

/* ---- Census without device allocation (no counterpart in the reference) ----
 * The census of IntermediateOutputAndCheck (src/CAupdate.cpp:738-808) computed over cell fields that
 * the caller holds in device memory, for callers that must not allocate device memory: a monitor
 * sampling solves that are still running (cudaMalloc / cudaFree may synchronise the device and
 * stall them) or a server whose HBM budget is fully handed out. It allocates nothing: its working
 * data lives in a fixed 26 KiB array in the library's device image (per device), which holds the
 * descriptors and accumulators of at most EXACA_CENSUS_MAX_DOMAINS domains per call; larger
 * n_domains returns EXACA_ERR_ARG. Each field pointer is a CUDA device pointer on `device`, indexed
 * like the pool's fields (k*mx*my + i*my + j); cell_type holds the reference's codes. */
#define EXACA_CENSUS_MAX_DOMAINS 256
typedef struct {
    const int8_t *cell_type;       /* domain_size cells */
    const int8_t *layer_id;        /* domain_size cells */
    const int32_t *crit_time_step; /* domain_size cells */
    int64_t domain_size;           /* cells */
    int64_t active_size;           /* cells of the active window (nzActive planes) */
    int32_t cycle;                 /* the CA cycle the census is taken at */
    int32_t layer;                 /* the current layer (layernumber): its cells are counted as
                                      superheated / undercooled / active / solid, liquid cells of
                                      other layers as remaining (src/CAupdate.cpp:741-757) */
    int64_t window_start;          /* first cell of the active window, ZBound_Low * mx * my: next_cts
                                      is taken over [window_start, window_start + active_size)
                                      (src/CAupdate.cpp:792-805) */
} exaca_cell_fields;
/* Writes out[i] for domains[i], i < n_domains, equal to what exaca_pool_census reports for a slot
 * holding the same fields at the same cycle. `stream` is a cudaStream_t (NULL: the legacy default
 * stream); the call waits for it before returning. The first call on a device looks up the scratch
 * array's device address and loads the kernel.
 * All calls on a device share the scratch array: a per-device lock keeps calls from several host
 * threads from overlapping on it. */
int exaca_census_cells(int device, void *stream, const exaca_cell_fields *domains, int n_domains, exaca_census *out);

#ifdef __cplusplus
}
#endif

#endif
