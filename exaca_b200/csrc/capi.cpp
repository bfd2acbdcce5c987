// C ABI of the B200 solver and the RunProgram_Reduced-equivalent driver (src/runCA.cpp:19-461).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>

#include "../../include/exaca_b200.h"
#include "exaca_host.hpp"
#include "pool.hpp"

struct exaca_problem {
    std::shared_ptr<exaca::Problem> p;
};
struct exaca_pool {
    std::unique_ptr<exaca::Pool> pool;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

template <class F> int guarded(F &&f) {
    try {
        f();
        return EXACA_OK;
    }
    catch (const std::invalid_argument &e) {
        return fail(EXACA_ERR_INPUT, std::string("invalid number in input: ") + e.what());
    }
    catch (const std::out_of_range &e) {
        return fail(EXACA_ERR_INPUT, std::string("number out of range in input: ") + e.what());
    }
    catch (const exaca::Unsupported &e) {
        return fail(EXACA_ERR_UNSUPPORTED, e.what());
    }
    catch (const exaca::AdmissionRefused &e) {
        return fail(EXACA_ERR_BUDGET, e.what());
    }
    catch (const exaca::DeviceError &e) {
        return fail(EXACA_ERR_CUDA, e.what());
    }
    catch (const std::bad_alloc &e) {
        return fail(EXACA_ERR_BUDGET, "host allocation failed");
    }
    catch (const std::exception &e) {
        return fail(EXACA_ERR_INPUT, e.what());
    }
    catch (...) {
        return fail(EXACA_ERR_INPUT, "unknown error");
    }
}

std::string fmt(double v) {
    std::ostringstream s;
    s << v;
    return s.str();
}

void emit(std::string &log) {
    std::cout << log << std::flush;
    log.clear();
}

void write_outputs(const exaca::Problem &p, const int32_t *gid, const std::string &prefix, std::string &log,
                   int threads = 0) {
    const exaca::InputConfig &c = p.cfg;
    if (c.print_misorientation || c.print_full_output) {
        log += "Collecting data on rank 0 and printing to files\n";
        if (c.print_misorientation) {
            log += "Printing Paraview file of grain misorientations\n";
            exaca::write_misorientations(p, gid, prefix + "_Misorientations.vtk", log, threads);
        }
        if (c.print_full_output) {
            log += "Printing layer ID, grain ID, and melted 0/1 data to a vtk file " + prefix +
                   ".vtk for post-processing\n";
            exaca::write_vtk_fields(p, gid, prefix + ".vtk", threads);
        }
    }
    else {
        log += "No output files to be printed, exiting program\n";
    }
}

} // namespace

namespace exaca {
void census_cells(int device, void *stream, const exaca_cell_fields *domains, int n_domains, exaca_census *out);
int census_device_count();
} // namespace exaca

extern "C" {

const char *exaca_last_error(void) { return g_last_error.c_str(); }

int exaca_problem_from_file(const char *input_file, exaca_problem **out) {
    if (!input_file || !out)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] {
        auto p = std::make_shared<exaca::Problem>();
        std::string log;
        exaca::read_input_file(input_file, p->cfg, log);
        exaca::initialize_problem(*p, log);
        *out = new exaca_problem{p};
    });
}

int exaca_problem_directional(const exaca_dirs_params *prm, exaca_problem **out) {
    if (!prm || !out)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] {
        auto p = std::make_shared<exaca::Problem>();
        exaca::InputConfig &c = p->cfg;
        // the values InputReadFromFile would produce for the equivalent type-C input file
        c.input_file = "<synthetic>";
        c.simulation_type = "C";
        c.decomposition_strategy = 1;
        c.material_name = "<synthetic>";
        c.A = prm->A;
        c.B = prm->B;
        c.C = prm->C;
        c.D = prm->D;
        c.freezing_range = prm->freezing_range;
        c.deltax = prm->cell_size_um * pow(10, -6);
        c.nread = prm->nucleation_density;
        c.nmax = c.nread * pow(10, 12);
        c.dTN = prm->dTN;
        c.dTsigma = prm->dTsigma;
        c.path_to_output = "./";
        c.output_file = "synthetic";
        std::string log;
        c.orientation_file = exaca::find_data_file("GrainOrientationVectors_Uniform10k.csv", "Substrate", log);
        c.number_of_layers = 1;
        c.G = prm->G;
        c.R = prm->R;
        c.nx = prm->nx + 2;
        c.ny = prm->ny + 2;
        c.nz = prm->nz + 2;
        c.deltat = c.deltax / (prm->n_ratio * (c.R / c.G));
        c.fract_surface_sites_active = prm->fract_surface_active;
        exaca::initialize_problem(*p, log);
        *out = new exaca_problem{p};
    });
}

void exaca_problem_free(exaca_problem *p) {
    if (p && p->p && p->p.use_count() == 1)
        exaca::unpin_problem(*p->p);
    delete p;
}

int exaca_problem_info(const exaca_problem *p, exaca_problem_geometry *info) {
    if (!p || !info)
        return fail(EXACA_ERR_ARG, "null argument");
    const exaca::Geometry &g = p->p->g;
    info->nx = g.nx;
    info->ny = g.ny;
    info->nz = g.nz;
    info->mx = g.mx;
    info->my = g.my;
    info->nz_active = g.nz_active;
    info->domain_size = g.domain_size;
    info->active_size = g.active_size;
    info->n_nuclei = (int)p->p->nuclei_loc.size();
    info->deltat = p->p->cfg.deltat;
    info->simulation_type = p->p->cfg.simulation_type.empty() ? '?' : p->p->cfg.simulation_type[0];
    return EXACA_OK;
}

int exaca_problem_fields(const exaca_problem *p, int32_t *cell_type, int32_t *grain_id, int32_t *cts, float *du,
                         int32_t *layer_id) {
    if (!p)
        return fail(EXACA_ERR_ARG, "null argument");
    const exaca::Problem &q = *p->p;
    int rc = guarded([&] { exaca::materialize_fields(q); });
    if (rc != EXACA_OK)
        return rc;
    long n = q.g.domain_size;
    for (long i = 0; i < n; i++) {
        if (cell_type)
            cell_type[i] = q.cell_type[i];
        if (grain_id)
            grain_id[i] = q.grain_id[i];
        if (cts)
            cts[i] = q.cts[i];
        if (du)
            du[i] = q.du[i];
        if (layer_id)
            layer_id[i] = q.layer_id[i];
    }
    return EXACA_OK;
}

int64_t exaca_problem_slot_bytes(const exaca_problem *p) { return p ? (int64_t)exaca::Pool::slot_bytes(*p->p) : -1; }

int exaca_pool_create(int device, size_t budget_bytes, uint64_t list_capacity, exaca_pool **out) {
    if (!out)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] { *out = new exaca_pool{std::make_unique<exaca::Pool>(device, budget_bytes, list_capacity)}; });
}

void exaca_pool_destroy(exaca_pool *pool) { delete pool; }

int exaca_pool_admit(exaca_pool *pool, const exaca_problem *p, int device_check, int *slot) {
    if (!pool || !p || !slot)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] { *slot = pool->pool->admit(p->p, device_check); });
}

int exaca_pool_step(exaca_pool *pool, int n_cycles) {
    if (!pool || n_cycles < 0)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] { pool->pool->step(n_cycles); });
}

int exaca_pool_status(exaca_pool *pool, int slot, exaca_domain_status *st) {
    if (!pool || !st || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] {
        pool->pool->sync_state();
        const exaca::DomainDesc &d = pool->pool->state(slot);
        st->cycle = d.cycle;
        st->done = d.done;
        st->nn = d.nn;
        st->error = d.error | pool->pool->pool_error();
        st->liquid = pool->pool->liquid(slot);
        st->layer = d.layer_no;
        st->window_z_lo = d.z_lo;
        st->window_nz = d.z_end - d.z_lo;
        st->reserved = 0;
    });
}

int exaca_pool_status_many(exaca_pool *pool, int n_slots, const int *slots, exaca_domain_status *st) {
    if (!pool || n_slots < 0 || (n_slots && (!slots || !st)))
        return fail(EXACA_ERR_ARG, "null argument");
    for (int i = 0; i < n_slots; i++)
        if (!pool->pool->slot_used(slots[i]))
            return fail(EXACA_ERR_ARG, "bad slot " + std::to_string(slots[i]));
    return guarded([&] {
        pool->pool->sync_state();
        const int perr = pool->pool->pool_error();
        for (int i = 0; i < n_slots; i++) {
            const exaca::DomainDesc &d = pool->pool->state(slots[i]);
            st[i].cycle = d.cycle;
            st[i].done = d.done;
            st[i].nn = d.nn;
            st[i].error = d.error | perr;
            st[i].liquid = pool->pool->liquid(slots[i]);
            st[i].layer = d.layer_no;
            st[i].window_z_lo = d.z_lo;
            st[i].window_nz = d.z_end - d.z_lo;
            st[i].reserved = 0;
        }
    });
}

int exaca_pool_grain_stats(exaca_pool *pool, int slot, const int32_t *region, exaca_grain_stats *out) {
    if (!pool || !out || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot or null argument");
    try {
        exaca::GrainStats g = pool->pool->grain_stats(slot, region);
        out->region_cells = g.region_cells;
        out->melted_cells = g.melted_cells;
        out->n_grains = g.n_grains;
        out->mean_grain_volume_um3 = g.deltax * g.deltax * pow(10, 12) * ((double)g.region_cells / (double)g.n_grains);
        out->nucleated_fraction = (double)g.nucleated_cells / (double)g.region_cells;
        out->mean_misorientation_deg = g.melted_cells ? g.misorientation_sum / (double)g.melted_cells : 0.0;
        out->mean_misorientation_top_deg = g.top_melted ? g.misorientation_top_sum / (double)g.top_melted : 0.0;
        for (int b = 0; b < exaca::kMisorientationBins; b++)
            out->misorientation_hist[b] = g.hist[b];
        return EXACA_OK;
    }
    catch (const std::invalid_argument &e) {
        return fail(EXACA_ERR_ARG, e.what());
    }
    catch (const std::exception &e) {
        return fail(EXACA_ERR_CUDA, e.what());
    }
}

int exaca_pool_stats(exaca_pool *pool, exaca_pool_stats_t *st) {
    if (!pool || !st)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] {
        exaca::PoolStats s = pool->pool->stats();
        st->cycles = s.cycles;
        st->launches = s.launches;
        st->listed = s.listed;
        st->grown = s.grown;
        st->captured = s.captured;
        st->nucleated = s.nucleated;
        st->claims = s.claims;
        st->row_reads = s.row_reads;
        st->dropped = s.dropped;
        st->fresh = s.fresh;
        st->rechecks = s.rechecks;
        st->flagged = s.flagged;
        st->h2d_bytes = s.h2d_bytes;
        st->d2h_bytes = s.d2h_bytes;
    });
}

double exaca_pool_last_run_ms(exaca_pool *pool) { return pool ? pool->pool->last_run_ms() : -1.0; }

int exaca_pool_profile_cycles(exaca_pool *pool, int n_cycles, double *kernel_ms) {
    if (!pool || !kernel_ms || n_cycles < 0)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] {
        exaca::KernelTimes t = pool->pool->profile_cycles(n_cycles);
        kernel_ms[0] = t.begin_ms;
        kernel_ms[1] = t.grow_ms;
        kernel_ms[2] = t.claim_ms;
        kernel_ms[3] = t.capture_ms;
    });
}

int exaca_pool_check_bounded_wait(exaca_pool *pool, int *flags) {
    if (!pool || !flags)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] { *flags = pool->pool->check_bounded_wait(); });
}

int exaca_pool_profile_persistent(exaca_pool *pool, int n_cycles, double *us) {
    if (!pool || !us || n_cycles < 0)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] { pool->pool->profile_persistent(n_cycles, us); });
}

int exaca_pool_run_all(exaca_pool *pool, int chunk_cycles, int64_t max_cycles, int64_t *cycles_stepped) {
    if (!pool || chunk_cycles <= 0 || max_cycles < 0)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] {
        long long n = pool->pool->run_all(chunk_cycles, max_cycles);
        if (cycles_stepped)
            *cycles_stepped = n;
    });
}

int exaca_pool_set_config(exaca_pool *pool, int config) {
    if (!pool || config < 0 || config >= exaca::Pool::kStepConfigs)
        return fail(EXACA_ERR_ARG, "step configuration out of range");
    return guarded([&] { pool->pool->set_config(config); });
}

int exaca_pool_set_grid(exaca_pool *pool, int divisor) {
    if (!pool || divisor < 0 || divisor > 32)
        return fail(EXACA_ERR_ARG, "grid divisor must be 0 (automatic) or 1-32");
    return guarded([&] { pool->pool->set_grid(divisor); });
}

int exaca_pool_autotune(exaca_pool *pool, int trial_cycles, int *config, double *ms_per_cycle) {
    if (!pool || trial_cycles <= 0)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] {
        int c = pool->pool->autotune(trial_cycles, ms_per_cycle);
        if (config)
            *config = c;
    });
}

int exaca_pool_timed_step(exaca_pool *pool, int n_cycles, double *ms) {
    if (!pool || !ms || n_cycles < 0)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] { *ms = pool->pool->timed_step(n_cycles); });
}

int exaca_problem_pin(exaca_problem *p) {
    if (!p)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] { exaca::pin_problem(*p->p); });
}

int exaca_pool_census(exaca_pool *pool, int slot, exaca_census *c) {
    if (!pool || !c || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] {
        pool->pool->sync_state();
        exaca::Census k = pool->pool->census(slot);
        c->superheated = k.superheated;
        c->undercooled = k.undercooled;
        c->active = k.active;
        c->solid = k.solid;
        c->remaining = k.remaining;
        c->next_cts = k.next_cts;
    });
}

int exaca_census_cells(int device, void *stream, const exaca_cell_fields *domains, int n_domains, exaca_census *out) {
    if (n_domains < 0 || n_domains > EXACA_CENSUS_MAX_DOMAINS)
        return fail(EXACA_ERR_ARG, "n_domains " + std::to_string(n_domains) + " outside 0.." +
                                       std::to_string(EXACA_CENSUS_MAX_DOMAINS) +
                                       " (the fixed census scratch holds at most that many domains)");
    if (n_domains == 0)
        return EXACA_OK;
    if (!domains || !out)
        return fail(EXACA_ERR_ARG, "null domains or out");
    for (int i = 0; i < n_domains; i++) {
        const exaca_cell_fields &d = domains[i];
        if (d.domain_size < 0 || d.active_size < 0 || d.window_start < 0 ||
            d.window_start > d.domain_size - d.active_size)
            return fail(EXACA_ERR_ARG,
                        "domain " + std::to_string(i) + ": bad domain_size / active_size / window_start");
        if (d.domain_size > 0 && (!d.cell_type || !d.layer_id || !d.crit_time_step))
            return fail(EXACA_ERR_ARG, "domain " + std::to_string(i) + ": null field pointer");
    }
    const int ndev = exaca::census_device_count();
    if (device < 0 || device >= ndev)
        return fail(EXACA_ERR_ARG, "bad device " + std::to_string(device));
    return guarded([&] { exaca::census_cells(device, stream, domains, n_domains, out); });
}

int exaca_pool_run_plain(exaca_pool *pool, int slot, int verbose, int *final_cycle) {
    if (!pool || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] {
        std::string log;
        int c = pool->pool->run_plain(slot, log, nullptr, nullptr);
        if (verbose)
            emit(log);
        if (final_cycle)
            *final_cycle = c;
    });
}

int exaca_pool_next_layer(exaca_pool *pool, int slot, int verbose) {
    if (!pool || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    const exaca::DomainDesc &d = pool->pool->state(slot);
    if (d.layer_no + 1 >= d.n_layers)
        return fail(EXACA_ERR_ARG, "slot " + std::to_string(slot) + " is in its last layer");
    return guarded([&] {
        std::string log;
        pool->pool->next_layer(slot, log);
        if (verbose)
            emit(log);
    });
}

int exaca_pool_copy_out(exaca_pool *pool, int slot, int32_t *grain_id, int32_t *cell_type) {
    if (!pool || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] {
        pool->pool->sync_state();
        pool->pool->copy_out(slot, grain_id, cell_type);
    });
}

int exaca_pool_copy_out_concurrent(exaca_pool *pool, int slot, int32_t *grain_id, int32_t *cell_type) {
    if (!pool || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] { pool->pool->copy_out_concurrent(slot, grain_id, cell_type); });
}

int exaca_pool_copy_octahedra(exaca_pool *pool, int slot, float *dl, float *doc, float *cdl) {
    if (!pool || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] {
        pool->pool->sync_state();
        pool->pool->copy_octahedra(slot, dl, doc, cdl);
    });
}

int exaca_pool_retire(exaca_pool *pool, int slot) {
    if (!pool || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad slot");
    return guarded([&] { pool->pool->retire(slot); });
}

int64_t exaca_pool_bytes_in_use(exaca_pool *pool) { return pool ? (int64_t)pool->pool->bytes_in_use() : -1; }

int exaca_pool_write_outputs(exaca_pool *pool, int slot, const exaca_problem *p, const char *path_prefix) {
    if (!pool || !p || !path_prefix || !pool->pool->slot_used(slot))
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] {
        std::vector<int32_t> gid(p->p->g.domain_size);
        pool->pool->copy_out(slot, gid.data(), nullptr);
        std::string log;
        write_outputs(*p->p, gid.data(), path_prefix, log);
        std::string out;
        exaca::RunTimes t;
        exaca::write_log(*p->p, std::string(path_prefix) + ".log", pool->pool->state(slot).cycle, t, out);
    });
}

int exaca_problem_write_outputs(const exaca_problem *p, const int32_t *grain_id, const char *path_prefix,
                                int threads) {
    if (!p || !grain_id || !path_prefix)
        return fail(EXACA_ERR_ARG, "bad argument");
    return guarded([&] {
        std::string log;
        write_outputs(*p->p, grain_id, path_prefix, log, threads);
    });
}

int exaca_run_program(const char *input_file, int device) {
    if (!input_file)
        return fail(EXACA_ERR_ARG, "null argument");
    return guarded([&] {
        // src/runCA.cpp:19-461 and src/main.cpp:15-47 at np = 1
        auto t_start = std::chrono::steady_clock::now();
        auto secs = [](std::chrono::steady_clock::time_point a) {
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        };
        std::string log = "ExaCA-B200: CUDA device " + std::to_string(device) + "\n";
        log += "Number of MPI ranks = 1\n";
        auto p = std::make_shared<exaca::Problem>();
        exaca::read_input_file(input_file, p->cfg, log);
        emit(log);
        exaca::initialize_problem(*p, log);
        emit(log);
        const exaca::Geometry &g = p->g;
        unsigned long long cap = (unsigned long long)g.active_size;
        exaca::Pool pool(device, (size_t)-1, cap);
        int slot = pool.admit(p, 0);
        exaca::RunTimes t;
        t.init = secs(t_start);
        log += "Data initialized: Time spent: " + fmt(t.init) + " s\n";
        emit(log);
        std::string prefix = p->cfg.path_to_output + p->cfg.output_file;
        if (p->cfg.print_debug) {
            std::vector<int32_t> gid(g.domain_size);
            pool.copy_out(slot, gid.data(), nullptr);
            exaca::materialize_fields(*p);
            exaca::Problem dbg = *p;
            dbg.grain_id = gid;
            log += "Printing initial data structures to a vtk file " + prefix + "_debug.vtk for debugging\n";
            exaca::write_debug_vtk(dbg, prefix + "_debug.vtk");
            log += "Initialization data file(s) printed\n";
            emit(log);
        }
        auto t_run = std::chrono::steady_clock::now();
        int cycle = pool.run_plain(slot, log, &t.nucl, &t.capture);
        t.run = secs(t_run);
        log += "Time for final layer was " + fmt(t.run) + " s\n";
        emit(log);
        auto t_out = std::chrono::steady_clock::now();
        std::vector<int32_t> gid(g.domain_size);
        pool.copy_out(slot, gid.data(), nullptr);
        write_outputs(*p, gid.data(), prefix, log);
        t.out = secs(t_out);
        log += "Printing ExaCA log file\n";
        exaca::write_log(*p, prefix + ".log", cycle, t, log);
        emit(log);
    });
}

} // extern "C"
