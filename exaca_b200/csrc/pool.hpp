// Device pool of ExaCA domains: the B200 runtime behind the C ABI.
//
// A pool owns a set of independent domains (one for the plain solver, hundreds for batched or
// served process maps). Every domain's fields live in their own HBM allocations; all domains share
// one compacted active-cell list, so one pass of the step kernels advances every admitted domain by
// one CA cycle; stretches of cycles run in one persistent cooperative launch.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "exaca_host.hpp"

namespace exaca {

constexpr int kMaxJumps = 32;
constexpr int kStepVariants = 4; // compiled launch shapes of the step passes
constexpr unsigned int kTombstone = 0xffffffffu;
constexpr unsigned int kNoRecord = 0xffffffffu;
constexpr int kLiquidShards = 16;
// Per-cycle counters that every warp reserves from are split into kShards counters (warp w uses
// shard w % kShards), each on its own 64-byte line, so their atomics do not queue on one address.
constexpr int kShards = 32;
struct alignas(64) ShardCounter {
    unsigned long long v;
    unsigned long long pad[7];
};
constexpr int kStatShards = 32;
// pool statistics, summed over shards
enum {
    kStatListed = 0,    // active-cell records visited
    kStatGrown = 1,     // records grown (eligible)
    kStatCaptured = 2,  // captures
    kStatNucleated = 3, // nucleation events
    kStatClaims = 4,    // atomicMin claims issued
    kStatRowReads = 5,  // critical-diagonal-length rows read (diagonal reached the cached minimum)
    kStatUnused = 6,
    kStatFresh = 7,     // liquid-neighbour masks built from the 26 neighbour types
    kStatRechecks = 8,  // solidification re-checks around claimed cells
    kStatDropped = 9,   // records dropped by the growth pass
    kStatFlagged = 10,  // records the growth pass handed to the claim pass
    kNumStats = 11
};

// One active cell in the compacted list: the state the per-cycle growth pass needs, so that pass
// streams 16-byte records instead of gathering per-cell arrays.
struct alignas(16) ActiveRec {
    float dl;          // DiagonalLength (dl and cdl_min form one aligned 8-byte pair)
    float cdl_min;     // lower bound of the critical lengths of the cell's liquid neighbours
    unsigned int cell; // index in the domain; kTombstone for a dropped record
    int cts;           // CritTimeStep
};
static_assert(sizeof(ActiveRec) == 16, "ActiveRec is one 16-byte vector");
static_assert(offsetof(ActiveRec, dl) % 8 == 0, "dl/cdl_min are stored as one float2");

// Device-resident descriptor of one domain. Static fields are written at admission; dynamic
// fields are advanced by the step kernels and read back by the host.
struct DomainDesc {
    // fields (index k*mx*my + i*my + j; the active window starts at k = 0 for single-layer problems)
    int8_t *ctype;
    int32_t *gid;
    int32_t *cts;
    int8_t *layer;
    float *du;
    float *dl;
    float *doc;               // 3 per active-window cell
    float *cdl;               // 26 per active-window cell
    unsigned long long *claim; // per active-window cell: (~epoch << 32) | capturer index
    unsigned int *pos;        // per active-window cell: position of its record in the list the next
                              // cycle reads (kNoRecord for cells that never had one)
    const double *growth;     // growth increment by number of undercooling updates
    const float *guv;         // 9 per orientation
    const float *cdl_table;   // 26 per orientation
    const int32_t *nuc_loc;   // nuclei sorted by nucleation time
    const int32_t *nuc_time;
    int growth_len;
    int n_nuclei;
    int mx, my, nz, nz_active, xoff, yoff, zbound_high;
    int check_mode; // 1: the device ends the domain at cycle % 1000 == 0 once no liquid is left
    long long domain_size, active_size;
    float du_value;
    int zero_du; // 1 if a cell that can become active has UndercoolingChange 0 (U stays 0 there)
    int cts_max; // check_mode domains: the largest CritTimeStep of any cell
    // dynamic state
    int cycle;
    unsigned int epoch;
    int nuc_cursor;
    int done;
    int nn;
    int error;
    int n_jumps;
    int dry_since; // check_mode domains past cts_max: the first cycle start that found no liquid (0: none)
    long long liquid; // liquid cells of layer 0, less the nucleations (captures are in liquid_shard)
    long long liquid_shard[kLiquidShards]; // minus the captures, spread over shards to avoid contention
    int jump_lo[kMaxJumps];
    int jump_hi[kMaxJumps];
    // Multilayer problems (src/runCA.cpp:282-411). cts_run is the CritTimeStep the step uses: the
    // cell's own for cells of the active window [z_lo, z_end) whose LayerID <= layer_no, INT_MAX
    // for every other cell (the reference's step does not touch them this layer). nu_base holds per
    // cell the undercooling updates of earlier layers (UndercoolingCurrent is never reset). For
    // single-layer problems cts_run == cts and nu_base is null.
    int32_t *cts_run;
    int32_t *nu_base;
    // Several UndercoolingChange values (type R): per cell the index of its growth table, which is
    // table du_class[cell] of growth (growth_len entries each). Null with one value.
    const uint16_t *du_class;
    int layer_no;
    int n_layers;
    int z_lo, z_end;
};

// Pool-level device state.
struct PoolState {
    ActiveRec *rec[2];           // active-cell records of the current / next cycle
    unsigned int *rdom[2];       // domain of each record
    unsigned int *rstat[2];      // per record: liquid-neighbour directions and flags (kMaskFresh: not built)
    // per record: (direction of the cached minimum critical length << 32) | second-smallest critical
    // length (float bits), both over the liquid neighbours not reached at the last claim step
    unsigned long long *rmin2[2];
    // claim queue: records the growth pass hands to the claim pass, with the state the claim needs;
    // shard s holds entries [s * shard_cap, s * shard_cap + qcnt_s[s])
    unsigned int *qpos, *qcell, *qdom, *qmask;
    float *qdl;
    // claims this cycle, (domain << 37) | (direction << 32) | claimed cell; shard s holds entries
    // [s * shard_cap, s * shard_cap + tcnt_s[s])
    unsigned long long *tgt;
    unsigned long long shard_cap;
    ShardCounter qcnt_s[kShards];
    ShardCounter tcnt_s[kShards];
    ShardCounter tomb_s[kShards]; // tombstones added this cycle (summed into tombs at the start of the next)
    unsigned long long cnt[2];
    unsigned long long capacity;
    unsigned long long tombs; // dropped records still in list `cur` (in-place cycles)
    int cur;                  // list read by this cycle's growth pass
    int pending;              // list the next cycle reads (cur, or cur ^ 1 when this cycle compacts)
    int compact;              // 1: this cycle's growth pass writes the survivors to list cur ^ 1
    int error;
    int n_domains;
    int extras; // 1 once a domain with per-cell growth extras (several layers or undercooling values) was admitted
    int claim_overflow; // 1: a block's claim queue overflowed this cycle, so the global claim pass runs
    int pad;
    DomainDesc *desc;
    unsigned long long stat[kStatShards][kNumStats];
    unsigned int blocks_done;      // last-block detection of the separate capture kernel
    unsigned int bar_count;        // grid-wide meeting point of the persistent kernel: arrivals
    unsigned int bar_gen;          // and generation
    unsigned long long *timeline;  // optional: per meeting point {first arrival, last arrival, release} (ns)
    unsigned long long work[2];    // spare counters
};

struct PoolStats {
    unsigned long long cycles; // CA cycles launched
    unsigned long long launches; // kernels launched by step()
    unsigned long long listed, grown, captured, nucleated, claims, row_reads, dropped, fresh, rechecks, flagged;
    unsigned long long h2d_bytes, d2h_bytes; // problem data copied host->device (fields or seeds, nuclei,
                                             // tables) and results copied back
};

// CUDA-event times of a stretch of cycles run pass by pass as separate kernels.
struct KernelTimes {
    double begin_ms = 0, grow_ms = 0, claim_ms = 0, capture_ms = 0;
    int cycles = 0;
};

// Result of the reference's every-1000-cycle census (src/CAupdate.cpp:738-808).
struct Census {
    unsigned long long superheated, undercooled, active, solid, remaining;
    unsigned long long next_cts; // min CritTimeStep of liquid cells in the active window
};

// Grain statistics of the reference analysis (analysis/src/GAprint.cpp:17-198) over one region.
constexpr int kMisorientationBins = 64;
struct GrainStats {
    long long region_cells = 0, melted_cells = 0, n_grains = 0, nucleated_cells = 0, top_melted = 0;
    double misorientation_sum = 0, misorientation_top_sum = 0, deltax = 0;
    unsigned long long hist[kMisorientationBins] = {};
};

struct DeviceTables {
    float *guv = nullptr;
    float *cdl_table = nullptr;
};

struct SlotHost {
    bool used = false;
    std::shared_ptr<const Problem> problem;
    std::vector<void *> allocs;
    double *growth = nullptr;
    int growth_len = 0;
    long long steps_launched = 0; // upper bound on executed updates of any cell of the slot
    size_t bytes = 0;
    int n_jumps = 0;
    bool finished = false;
};

class Pool {
  public:
    Pool(int device, size_t budget_bytes, unsigned long long list_capacity);
    ~Pool();
    Pool(const Pool &) = delete;
    Pool &operator=(const Pool &) = delete;

    // HBM bytes a problem needs in a pool slot.
    static size_t slot_bytes(const Problem &p);
    // Uploads an initialised problem; returns the slot index. check_mode 1 lets the device end
    // the domain on its own; 0 leaves termination to run_plain's host-side census.
    int admit(std::shared_ptr<const Problem> p, int check_mode);
    void retire(int slot);
    // Advances every unfinished domain by n cycles (one persistent cooperative launch).
    void step(int n);
    // Reads back the dynamic state of all slots.
    void sync_state();
    const DomainDesc &state(int slot) const { return host_desc_.at(slot); }
    Census census(int slot);
    void copy_out(int slot, int32_t *grain_id, int32_t *cell_type);
    void copy_out_raw(int slot, int32_t *grain_id, int8_t *cell_type);
    // copy_out of a slot whose domain has ended (as of the last state read) on a separate copy
    // stream: it does not wait for cycles launched since, so a request loop can copy finished
    // results while the next cycles run. Returns when the data is on the host.
    void copy_out_concurrent(int slot, int32_t *grain_id, int32_t *cell_type);
    void copy_octahedra(int slot, float *dl, float *doc, float *cdl);
    // One device-to-host transfer of to_host: bytes from device memory src to host dst, or with
    // widen bytes int8 values to int32 at dst. A null dst is skipped.
    struct HostCopy {
        void *dst;
        const void *src;
        size_t bytes;
        bool widen;
    };
    // Issues the transfers on stream (a cudaStream_t) after the work already queued there and
    // returns when every pageable destination holds its data; page-locked destinations take one
    // DMA each, still in flight at return. Pageable ones go through two 32 MB pinned staging
    // pieces, the DMA of one overlapping the multi-threaded move out of the other: the driver's
    // own pageable path moves about 2 GB/s.
    void to_host(const std::vector<HostCopy> &copies, void *stream);
    // writes the diagonal lengths held in the active records back to the per-cell array
    void flush_records();
    // Reference-equivalent run of one slot to completion with the reference's 1000-cycle census,
    // stdout progress lines, type-S cycle jumps and, for multilayer problems, the move of the active
    // window between layers (src/runCA.cpp:282-411).
    int run_plain(int slot, std::string &log, double *nucl_s, double *capture_s);
    // Ends the current layer of a multilayer slot and sets up the next one: DomainShiftAndResize
    // and LayerSetup (src/CAinitialize.cpp:2772-2982). Appends the reference's lines to `log`.
    void next_layer(int slot, std::string &log);
    // device time (CUDA events on the pool stream) of the last run_plain
    double last_run_ms() const { return last_run_ms_; }
    // runs n cycles as separate per-pass kernels with CUDA events around each launch
    KernelTimes profile_cycles(int n);
    // Grain statistics of a slot's GrainID field over a region in .vtk coordinates
    // {xmin, xmax, ymin, ymax, zmin, zmax} (null: the interior without wall layers).
    GrainStats grain_stats(int slot, const int *region);
    // step(n) with CUDA events around the launches; returns their device time in ms
    double timed_step(int n);
    // Step configurations: config = mode * kStepVariants + variant. set_config switches; autotune
    // runs trial_cycles real cycles with every configuration (the pool's domains advance), keeps
    // the fastest and returns it; ms_per_cycle (kStepConfigs entries, may be null) gets the trials.
    // Either fixes the configuration for run_plain, which otherwise picks the fastest persistent
    // one itself (plain_tune).
    static constexpr int kStepConfigs = 2 * kStepVariants;
    void set_config(int config);
    // Persistent grid: 0 chooses itself (run_plain's trials, else the list length), 1 all co-resident
    // blocks, 2 half of them.
    void set_grid(int divisor);
    int config() const { return step_mode_ * kStepVariants + variant_; }
    int autotune(int trial_cycles, double *ms_per_cycle);
    // Steps every admitted domain in chunks of `chunk` cycles until each one has ended on the device
    // (admitted with check_mode 1); returns the cycles stepped. Throws past max_cycles.
    long long run_all(int chunk, long long max_cycles);
    // step(n) with the persistent kernel's timeline on; per-cycle averages in microseconds of
    // {growth pass: first block done, last block done; claim pass: first, last; capture pass: first,
    // last; end of cycle and start of the next (last block alone)}
    void profile_persistent(int n, double us[7]);
    int n_slots() const { return (int)slots_.size(); }
    bool slot_used(int s) const { return s < (int)slots_.size() && slots_[s].used; }
    size_t bytes_in_use() const { return bytes_in_use_; }
    size_t budget() const { return budget_; }
    int device() const { return device_; }
    unsigned long long list_count();
    PoolStats stats();
    long long liquid(int slot) const;
    void set_cycle(int slot, int cycle);
    int pool_error();
    // Runs the persistent kernel's grid-wide wait where nothing can release it; returns the pool
    // error flags it left (kErrBarrier after the 1 s limit) and clears them.
    int check_bounded_wait();

  private:
    void ensure_growth(int slot, long long needed);
    void push_desc(int slot);
    void launch_persistent(int n);
    void launch_passes(int n); // n cycles as separate pass kernels (stream order)
    void build_graph();
    const DeviceTables &tables_for(const Problem &p);

    int device_;
    size_t budget_;
    size_t bytes_in_use_ = 0;
    void *stream_ = nullptr;      // cudaStream_t
    void *copy_stream_ = nullptr; // cudaStream_t of copy_out_concurrent (created on first use)
    void *stage_[2] = {nullptr, nullptr};    // to_host's pinned staging pieces (first use)
    void *stage_ev_[2] = {nullptr, nullptr}; // cudaEvent_t marking each piece's DMA
    PoolState *dstate_ = nullptr;
    DomainDesc *ddesc_ = nullptr;
    int max_domains_ = 0;
    int n_domains_ = 0; // highest used slot + 1 (mirrors PoolState::n_domains)
    unsigned long long capacity_ = 0;
    std::vector<SlotHost> slots_;
    std::vector<DomainDesc> host_desc_;
    std::map<std::string, DeviceTables> tables_;
    int num_sms_ = 148;
    unsigned long long cycles_launched_ = 0;
    // step configuration: mode (0: persistent kernel, 1: CUDA graph of the separate pass kernels)
    // x launch-shape variant (kStepVariants compiled lane / batch combinations)
    int step_mode_ = 0;
    int variant_ = kStepVariants - 1;
    bool config_fixed_ = false; // set_config or autotune chose the configuration
    // Persistent grid: all co-resident blocks (grid_div_ 1) or half of them (2), which cuts the
    // grid-wide meetings' cost when the list is short. run_plain's trials choose it; otherwise it
    // follows the list length read at the last sync_state.
    int grid_div_ = 1;
    bool grid_tuned_ = false;
    bool plain_run_ = false; // inside run_plain
    int grid_fixed_ = 0; // set_grid's divisor, 0 when the grid chooses itself
    unsigned long long last_records_ = 0;
    void apply_config(int config);
    // run_plain's choice: n real cycles with each persistent configuration (and grid), the fastest
    // kept; returns the cycles run
    int plain_tune(int n);
    int grid_cycles_[kStepVariants] = {}; // co-resident blocks of each persistent kernel
    int grid_grow_[kStepVariants] = {};
    int grid_capture_[kStepVariants] = {};
    void *graph_exec_ = nullptr;
    int graph_steps_ = 0;
    int grid_claim_ = 0;
    unsigned long long launches_ = 0;
    unsigned long long h2d_bytes_ = 0, d2h_bytes_ = 0;
    double last_run_ms_ = 0;
    void *census_buf_ = nullptr;
};

} // namespace exaca
