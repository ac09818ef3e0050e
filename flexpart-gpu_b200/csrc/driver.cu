// driver.cu — the forward time loop (ForwardTimeLoopDriver,
// src/simulation/timeloop.rs:660-1431) and the release manager
// (src/release/mod.rs:55-275) as host C++ over the fpg.h entry points.
//
// Host bookkeeping mirrors ParticleStore (src/particles/mod.rs:477-605):
// slots are handed out from the lowest free index; nothing on the device
// deactivates a particle, so the free slots are always [next_free, capacity)
// (after a compaction: [active_count, capacity), reset_after_compaction).
//
// Launch range and Philox counters: the reference dispatches every capacity
// slot and advances the counter by dispatch_count * blocks per step
// (gpu/langevin_fused.rs:229-233); slots at or above next_free are zeroed
// (inactive) and their kernels return at once.  The driver launches only
// [0, next_free) and advances the counter by the reference's dispatch count,
// so every particle draws the same Philox blocks as in the reference.
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/fpg_driver.h"
#include "fpg_internal.h"

namespace {

struct ReleaseState {
    fpg_release cfg;
    uint64_t released = 0;
    int32_t release_point = 0;
};

int64_t days_from_civil(int64_t y, int64_t m, int64_t d) {
    if (m <= 2) y -= 1;
    const int64_t era = (y >= 0 ? y : y - 399) / 400;
    const int64_t yoe = y - era * 400;
    const int64_t mp = m + (m > 2 ? -3 : 9);
    const int64_t doy = (153 * mp + 2) / 5 + d - 1;
    const int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + doe - 719468;
}

// ReleaseState::target_emitted_count (release/mod.rs:181-196).
uint64_t target_emitted(const ReleaseState& s, int64_t now) {
    const fpg_release& r = s.cfg;
    if (now < r.start_seconds || now > r.end_seconds) return s.released;
    if (r.start_seconds == r.end_seconds) return r.particle_count;
    if (now == r.end_seconds) return r.particle_count;
    const unsigned __int128 e = (uint64_t)(now - r.start_seconds);
    const unsigned __int128 d = (uint64_t)(r.end_seconds - r.start_seconds);
    return (uint64_t)(((unsigned __int128)r.particle_count * e) / d);
}

// ReleaseBounds::sample_stratified (release/mod.rs:256-275).
void sample_stratified(const fpg_release& r, uint64_t index, uint64_t total, double& lon, double& lat, double& z) {
    double c = std::ceil(std::cbrt((double)total));
    if (c < 1.0) c = 1.0;
    const uint64_t nx = (uint64_t)c, ny = nx;
    uint64_t nxy = nx * ny;
    if (nxy < 1) nxy = 1;
    uint64_t nz = (total + nxy - 1) / nxy;
    if (nz < 1) nz = 1;
    const uint64_t ix = index % nx, iy = (index / nx) % ny, iz = (index / nxy) % nz;
    const double fx = ((double)ix + 0.5) / (double)nx;
    const double fy = ((double)iy + 0.5) / (double)ny;
    const double fz = ((double)iz + 0.5) / (double)nz;
    lon = r.lon_min + fx * (r.lon_max - r.lon_min);
    lat = r.lat_min + fy * (r.lat_max - r.lat_min);
    z = r.z_min + fz * (r.z_max - r.z_min);
}

}  // namespace

struct fpg_forward {
    fpg_ctx* ctx = nullptr;
    fpg_forward_config cfg{};
    fpg_grid_domain domain{};
    std::vector<ReleaseState> releases;
    size_t capacity = 0;
    fpg_particles* particles = nullptr;
    fpg_met* met = nullptr;
    fpg_surface* surface = nullptr;
    fpg_pbl* pbl = nullptr;
    fpg_compaction* compaction = nullptr;
    fpg_sorter* sorter = nullptr;
    int64_t t = 0;
    uint64_t step_index = 0;
    uint32_t counter[4] = {0, 0, 0, 0};
    size_t next_free = 0;
    size_t active = 0;
    bool have_bracket = false;
    int64_t bracket_t0 = 0, bracket_t1 = 0;
    float* d_forcing[3] = {nullptr, nullptr, nullptr};   // dry velocity, wet lambda, wet fraction per slot
    std::vector<fpg_particle> staging;
    // +1 forward; -1 backward (BackwardTimeLoopDriver): the clock runs back,
    // advection takes -dt and turbulence/deposition +dt (timeloop.rs:1724-1746)
    int direction = 1;
    // met streaming: frames copied ahead on copy_stream into ring slots
    struct MetSlot {
        int64_t time = 0;
        bool valid = false;
        uint64_t last_use = 0;
        float* uvw = nullptr;                 // 3 * nodes
        fpg_surface_cell* surface = nullptr;  // nx * ny
        cudaEvent_t copied = nullptr;         // recorded on copy_stream after the copy
        cudaEvent_t released = nullptr;       // recorded on the step stream after the last read
    };
    std::vector<MetSlot> ring;
    cudaStream_t copy_stream = nullptr;
    uint64_t tick = 0, ring_hits = 0, host_uploads = 0;
    // per-section timing (fpg_forward_set_profiling / FLEXPART_GPU_PROFILE=1)
    bool profile = false, print_profile = false, have_timing = false;
    cudaEvent_t marks[7] = {};
    fpg_step_timing last_timing{};
    // validation mode (fpg_forward_set_validation_mode / FLEXPART_GPU_VALIDATION=1):
    // separated passes with a per-slot Hanna record buffer (capacity records)
    bool validation = false;
    fpg_hanna_params* hanna_records = nullptr;
};

namespace {

// One NVTX range (a named span in Nsight timelines; nothing without a tool).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { end(); }
    void end() {
        if (open) nvtxRangePop();
        open = false;
    }
    bool open = true;
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Records section boundary k on the step stream when timing is on.
void mark(fpg_forward* d, int k) {
    if (d->profile) cudaEventRecord(d->marks[k], d->ctx->stream);
}

fpg_status ensure_marks(fpg_forward* d) {
    for (cudaEvent_t& e : d->marks)
        if (!e) FPG_CUDA(cudaEventCreate(&e));
    return FPG_OK;
}

}  // namespace

using namespace fpg;

extern "C" void fpg_forward_config_default(fpg_forward_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->start_seconds = 1704067200;   // 20240101000000
    c->end_seconds = 1704067200;
    c->timestep_seconds = 1;
    c->clamp_time_bounds = 1;
    c->x_grid_per_meter = c->y_grid_per_meter = c->z_grid_per_meter = 1.0f;
    c->pbl_options = fpg_pbl_options{0.1f, 10.0f, 1.0f, 800.0f, 100.0f, 4500.0f};
    c->dry_reference_height_m = 15.0f;
    c->philox_key[0] = 0xDECAFBADu;
    c->philox_key[1] = 0x12345678u;
    c->sort_interval_steps = 0;
    c->use_compaction = 0;
    c->n_substeps = 4;
    c->min_height_m = 0.01f;
}

extern "C" fpg_status fpg_parse_timestamp(const char* s, int64_t* out) {
    if (!s || !out || std::strlen(s) != 14) return FPG_ERR_INVALID_ARGUMENT;
    int v[14];
    for (int i = 0; i < 14; ++i) {
        if (s[i] < '0' || s[i] > '9') return FPG_ERR_INVALID_ARGUMENT;
        v[i] = s[i] - '0';
    }
    const int64_t year = v[0] * 1000 + v[1] * 100 + v[2] * 10 + v[3];
    const int64_t month = v[4] * 10 + v[5], day = v[6] * 10 + v[7];
    const int64_t hour = v[8] * 10 + v[9], minute = v[10] * 10 + v[11], second = v[12] * 10 + v[13];
    if (month < 1 || month > 12 || day < 1 || day > 31 || hour > 23 || minute > 59 || second > 59)
        return FPG_ERR_INVALID_ARGUMENT;
    *out = days_from_civil(year, month, day) * 86400 + hour * 3600 + minute * 60 + second;
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_destroy(fpg_forward* d) {
    if (!d) return FPG_OK;
    fpg_ctx_synchronize(d->ctx, nullptr);
    fpg_particles_destroy(d->particles);
    fpg_met_destroy(d->met);
    fpg_surface_destroy(d->surface);
    fpg_pbl_destroy(d->pbl);
    fpg_compaction_destroy(d->compaction);
    fpg_sorter_destroy(d->sorter);
    for (float* p : d->d_forcing) cudaFree(p);
    for (auto& slot : d->ring) {
        cudaFree(slot.uvw);
        cudaFree(slot.surface);
        if (slot.copied) cudaEventDestroy(slot.copied);
        if (slot.released) cudaEventDestroy(slot.released);
    }
    if (d->copy_stream) {
        cudaStreamSynchronize(d->copy_stream);
        cudaStreamDestroy(d->copy_stream);
    }
    for (cudaEvent_t e : d->marks)
        if (e) cudaEventDestroy(e);
    cudaFree(d->hanna_records);
    delete d;
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_set_profiling(fpg_forward* d, int32_t on) {
    if (!d) return FPG_ERR_INVALID_ARGUMENT;
    if (on) {
        const fpg_status st = ensure_marks(d);
        if (st != FPG_OK) return st;
    }
    d->profile = on != 0;
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_set_validation_mode(fpg_forward* d, int32_t on) {
    if (!d) return FPG_ERR_INVALID_ARGUMENT;
    if (on && !d->hanna_records)
        FPG_CUDA(cudaMalloc(&d->hanna_records, (d->capacity > 0 ? d->capacity : 1) * sizeof(fpg_hanna_params)));
    d->validation = on != 0;
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_last_timing(const fpg_forward* d, fpg_step_timing* out) {
    if (!d || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (!d->have_timing) return FPG_ERR_NOT_READY;
    *out = d->last_timing;
    return FPG_OK;
}

static fpg_status driver_create(fpg_ctx* ctx, const fpg_forward_config* cfg, const fpg_release* rel, size_t n_rel,
                                const fpg_grid_domain* grid, size_t capacity, size_t nx, size_t ny, size_t nz,
                                const float* heights, int direction, fpg_forward** out);

extern "C" fpg_status fpg_forward_create(fpg_ctx* ctx, const fpg_forward_config* cfg, const fpg_release* rel,
                                         size_t n_rel, const fpg_grid_domain* grid, size_t capacity, size_t nx,
                                         size_t ny, size_t nz, const float* heights, fpg_forward** out) {
    if (!ctx || !cfg || !grid || !out || (n_rel && !rel)) return FPG_ERR_INVALID_ARGUMENT;
    // validate_config (timeloop.rs:1932-1972)
    if (cfg->start_seconds > cfg->end_seconds) return FPG_ERR_INVALID_TIME_RANGE;
    return driver_create(ctx, cfg, rel, n_rel, grid, capacity, nx, ny, nz, heights, 1, out);
}

static fpg_status driver_create(fpg_ctx* ctx, const fpg_forward_config* cfg, const fpg_release* rel, size_t n_rel,
                                const fpg_grid_domain* grid, size_t capacity, size_t nx, size_t ny, size_t nz,
                                const float* heights, int direction, fpg_forward** out) {
    if (cfg->timestep_seconds <= 0) return FPG_ERR_INVALID_TIME_STEP;
    if (!std::isfinite(cfg->dry_reference_height_m) || cfg->dry_reference_height_m <= 0.0f)
        return FPG_ERR_INVALID_REFERENCE_HEIGHT;
    // ReleaseBounds::from_config (release/mod.rs:221-244)
    for (size_t i = 0; i < n_rel; ++i)
        if (rel[i].lon_min > rel[i].lon_max || rel[i].lat_min > rel[i].lat_max || rel[i].z_min > rel[i].z_max)
            return FPG_ERR_INVALID_BOUNDS;
    fpg_forward* d = new fpg_forward();
    d->ctx = ctx;
    d->cfg = *cfg;
    d->direction = direction;
    d->domain = *grid;
    d->capacity = capacity;
    d->t = cfg->start_seconds;
    std::memcpy(d->counter, cfg->initial_philox_counter, sizeof(d->counter));
    for (size_t i = 0; i < n_rel; ++i) {
        ReleaseState s;
        s.cfg = rel[i];
        s.release_point = (int32_t)i;
        d->releases.push_back(s);
    }
    fpg_status st = fpg_particles_create(ctx, capacity, &d->particles);
    if (st == FPG_OK) st = fpg_met_create(ctx, nx, ny, nz, &d->met);
    if (st == FPG_OK && heights) st = fpg_met_set_level_heights(d->met, heights, nz);
    if (st == FPG_OK) st = fpg_surface_create(ctx, nx, ny, &d->surface);
    if (st == FPG_OK) st = fpg_pbl_create(ctx, nx, ny, &d->pbl);
    // is_compaction_enabled (timeloop.rs:496-513): FLEXPART_GPU_COMPACTION=1 turns
    // compaction on as the configuration's use_compaction does
    const char* cmp = std::getenv("FLEXPART_GPU_COMPACTION");
    const bool compaction = cfg->use_compaction || (cmp && std::strcmp(cmp, "1") == 0);
    if (st == FPG_OK && compaction) st = fpg_compaction_create(ctx, capacity, &d->compaction);
    if (st == FPG_OK && cfg->sort_interval_steps) st = fpg_sorter_create(ctx, capacity, &d->sorter);
    // is_profiling_enabled (timeloop.rs:469-476)
    const char* prof = std::getenv("FLEXPART_GPU_PROFILE");
    if (st == FPG_OK && prof && std::strcmp(prof, "1") == 0) {
        st = fpg_forward_set_profiling(d, 1);
        d->print_profile = true;
    }
    // is_validation_mode (timeloop.rs:480-494)
    const char* val = std::getenv("FLEXPART_GPU_VALIDATION");
    if (st == FPG_OK && val && std::strcmp(val, "1") == 0) st = fpg_forward_set_validation_mode(d, 1);
    if (st != FPG_OK) {
        fpg_forward_destroy(d);
        return st;
    }
    *out = d;
    return FPG_OK;
}

extern "C" int32_t fpg_forward_has_remaining_steps(const fpg_forward* d) {
    if (!d) return 0;
    return d->direction > 0 ? d->t <= d->cfg.end_seconds : d->t >= d->cfg.end_seconds;
}
extern "C" int64_t fpg_forward_current_time(const fpg_forward* d) { return d ? d->t : 0; }
extern "C" fpg_particles* fpg_forward_particles(fpg_forward* d) { return d ? d->particles : nullptr; }

extern "C" fpg_status fpg_forward_finalize(fpg_forward* d) {
    if (!d) return FPG_ERR_INVALID_ARGUMENT;
    return fpg_ctx_synchronize(d->ctx, nullptr);
}

// ReleaseManager::inject_for_time + upload of the touched slots
// (release/mod.rs:90-168).
static fpg_status release_for_time(fpg_forward* d, int64_t now, uint64_t& released, uint64_t& first_slot) {
    released = 0;
    first_slot = d->next_free;
    d->staging.clear();
    for (ReleaseState& s : d->releases) {
        const uint64_t target = target_emitted(s, now);
        if (target <= s.released) continue;
        const uint64_t to_emit = target - s.released;
        const float mass_per_particle = (float)(s.cfg.mass_kg / (double)s.cfg.particle_count);
        for (uint64_t k = 0; k < to_emit; ++k) {
            double lon, lat, z;
            sample_stratified(s.cfg, s.released + k, s.cfg.particle_count, lon, lat, z);
            // geo_to_grid, GridDomain::contains, GridCoord::to_relative (coords/mod.rs:92-114,169-178)
            const double x = (lon - d->domain.xlon0) / d->domain.dx;
            const double y = (lat - d->domain.ylat0) / d->domain.dy;
            if (!(x >= 0.0 && x < (double)(d->domain.nx - 1) && y >= 0.0 && y < (double)(d->domain.ny - 1)))
                return FPG_ERR_OUT_OF_GRID;
            if (d->next_free + d->staging.size() >= d->capacity) return FPG_ERR_STORE_FULL;
            const double fx = std::floor(x), fy = std::floor(y);
            fpg_particle p;
            std::memset(&p, 0, sizeof(p));
            p.cell_x = (int32_t)fx;
            p.cell_y = (int32_t)fy;
            p.pos_x = (float)(x - fx);
            p.pos_y = (float)(y - fy);
            p.pos_z = (float)z;
            p.flags = FPG_FLAG_ACTIVE;
            p.mass[0] = mass_per_particle;
            p.time = (int32_t)now;
            p.time_mem = (int32_t)now;
            p.release_point = s.release_point;
            d->staging.push_back(p);
        }
        s.released = target;
    }
    if (d->staging.empty()) return FPG_OK;
    const fpg_status st = fpg_particles_upload(d->particles, d->next_free, d->staging.size(), d->staging.data(),
                                               nullptr);
    if (st != FPG_OK) return st;
    released = d->staging.size();
    d->next_free += released;
    d->active += released;
    return FPG_OK;
}

static fpg_status upload_forcing(fpg_forward* d, int k, const float* host) {
    if (!d->d_forcing[k]) FPG_CUDA(cudaMalloc(&d->d_forcing[k], (d->capacity > 0 ? d->capacity : 1) * sizeof(float)));
    FPG_CUDA(cudaMemcpyAsync(d->d_forcing[k], host, d->capacity * sizeof(float), cudaMemcpyHostToDevice,
                             d->ctx->stream));
    return FPG_OK;
}

// The ring slot holding the frame valid at time t, or -1.
static int ring_find(const fpg_forward* d, int64_t t) {
    for (size_t i = 0; i < d->ring.size(); ++i)
        if (d->ring[i].valid && d->ring[i].time == t) return (int)i;
    return -1;
}

// Both frames of bracket (t0, t1) from the ring, packed on the step stream
// after their copies; FPG_ERR_NOT_READY when either is missing.
static fpg_status bracket_from_ring(fpg_forward* d, int64_t t0, int64_t t1) {
    const int i0 = ring_find(d, t0), i1 = ring_find(d, t1);
    if (i0 < 0 || i1 < 0) return FPG_ERR_NOT_READY;
    cudaStream_t s = d->ctx->stream;
    const size_t nodes = d->met->nx * d->met->ny * d->met->nz, cells = d->met->nx * d->met->ny;
    const int idx[2] = {i0, i1};
    for (int which = 0; which < 2; ++which) FPG_CUDA(cudaStreamWaitEvent(s, d->ring[idx[which]].copied, 0));
    const float* f0 = d->ring[i0].uvw;
    const float* f1 = d->ring[i1].uvw;
    fpg_status st = fpg_met_upload_bracket_device(d->met, f0, f0 + nodes, f0 + 2 * nodes, f1, f1 + nodes,
                                                  f1 + 2 * nodes, nullptr);
    if (st != FPG_OK) return st;
    for (int which = 0; which < 2; ++which) {
        fpg_forward::MetSlot& slot = d->ring[idx[which]];
        FPG_CUDA(cudaMemcpyAsync(d->surface->frame[which], slot.surface, cells * sizeof(fpg_surface_cell),
                                 cudaMemcpyDeviceToDevice, s));
        d->surface->uploaded[which] = true;
        slot.last_use = ++d->tick;
    }
    // the slots are not read after the repack: later copies into them wait for this
    for (int which = 0; which < 2; ++which) FPG_CUDA(cudaEventRecord(d->ring[idx[which]].released, s));
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_run_timestep(fpg_forward* d, const fpg_met_bracket* met, const fpg_forcing* f,
                                               fpg_step_report* report) {
    if (!d || !met || !f) return FPG_ERR_INVALID_ARGUMENT;
    if (!fpg_forward_has_remaining_steps(d)) return FPG_ERR_SIMULATION_COMPLETE;
    fpg_status st;
    const auto host_t0 = std::chrono::steady_clock::now();
    NvtxRange step_range("fpg step");
    mark(d, 0);

    // apply_spatial_sort_if_enabled (timeloop.rs:1414-1430)
    if (d->sorter && d->step_index % d->cfg.sort_interval_steps == 0 && d->next_free > 0) {
        NvtxRange r("reorder");
        const size_t keep = d->particles->dispatch;
        d->particles->dispatch = d->next_free;
        st = fpg_sort_by_cell(d->ctx, d->particles, d->met, d->sorter, nullptr, nullptr);
        d->particles->dispatch = keep;
        if (st != FPG_OK) return st;
    }
    mark(d, 1);

    uint64_t released = 0, first_slot = 0;
    {
        NvtxRange r("release");
        st = release_for_time(d, d->t, released, first_slot);
    }
    if (st != FPG_OK) return st;
    mark(d, 2);
    NvtxRange bracket_range("met bracket");

    // interpolation_alpha (timeloop.rs:2086-2120)
    const int64_t t0 = met->time_t0_seconds, t1 = met->time_t1_seconds;
    if (t1 <= t0) return FPG_ERR_INVALID_BRACKET;
    int64_t eff = d->t;
    if (!(d->t >= t0 && d->t <= t1)) {
        if (!d->cfg.clamp_time_bounds) return FPG_ERR_OUTSIDE_BRACKET;
        eff = d->t < t0 ? t0 : t1;
    }
    const float alpha = (float)((double)(eff - t0) / (double)(t1 - t0));

    // upload_dual_wind_if_bracket_changed (timeloop.rs:1378-1402) + surface frames
    if (!d->have_bracket || d->bracket_t0 != t0 || d->bracket_t1 != t1) {
        if ((st = bracket_from_ring(d, t0, t1)) == FPG_OK) {
            d->ring_hits += 1;
            d->have_bracket = true;
            d->bracket_t0 = t0;
            d->bracket_t1 = t1;
        } else if (st != FPG_ERR_NOT_READY) {
            return st;
        }
    }
    if (!d->have_bracket || d->bracket_t0 != t0 || d->bracket_t1 != t1) {
        d->host_uploads += 1;
        if (!met->wind_t0_u || !met->wind_t0_v || !met->wind_t0_w || !met->wind_t1_u || !met->wind_t1_v ||
            !met->wind_t1_w || !met->surface_t0 || !met->surface_t1)
            return FPG_ERR_INVALID_ARGUMENT;
        if ((st = fpg_met_upload_frame(d->met, 0, met->wind_t0_u, met->wind_t0_v, met->wind_t0_w, nullptr))) return st;
        if ((st = fpg_met_upload_frame(d->met, 1, met->wind_t1_u, met->wind_t1_v, met->wind_t1_w, nullptr))) return st;
        if ((st = fpg_surface_upload(d->surface, 0, met->surface_t0, nullptr))) return st;
        if ((st = fpg_surface_upload(d->surface, 1, met->surface_t1, nullptr))) return st;
        d->have_bracket = true;
        d->bracket_t0 = t0;
        d->bracket_t1 = t1;
    }
    bracket_range.end();
    mark(d, 3);
    // interpolate_surface_fields_linear + encode_pbl_diagnostics (timeloop.rs:961-988,1079-1088)
    {
        NvtxRange r("pbl");
        if ((st = fpg_pbl_diagnostics(d->ctx, d->surface, alpha, &d->cfg.pbl_options, d->pbl, nullptr))) return st;
    }
    mark(d, 4);
    NvtxRange step_kernel_range("fused step");

    // the fused step (timeloop.rs:1095-1180)
    const float dt = (float)d->cfg.timestep_seconds;
    fpg_step_params p;
    fpg_step_params_default(&p);
    p.alpha = alpha;
    p.dt_seconds = d->direction > 0 ? dt : -dt;   // TimeDirection::advection_dt_seconds (timeloop.rs:137-142)
    p.turb_dt_seconds = dt;
    p.x_grid_per_meter = d->cfg.x_grid_per_meter;
    p.y_grid_per_meter = d->cfg.y_grid_per_meter;
    p.z_grid_per_meter = d->cfg.z_grid_per_meter;
    p.n_substeps = d->cfg.n_substeps;
    p.min_height_m = d->cfg.min_height_m;
    p.rho_grad_over_rho = f->rho_grad_over_rho;
    p.key[0] = d->cfg.philox_key[0];
    p.key[1] = d->cfg.philox_key[1];
    std::memcpy(p.counter, d->counter, sizeof(p.counter));
    p.dry_reference_height_m = d->cfg.dry_reference_height_m;
    // is_zero(): Uniform(0) skips the process (timeloop.rs:998-1000)
    p.dry_mode = (f->dry_mode == FPG_FORCING_UNIFORM && f->dry_velocity_m_s == 0.0f) ? FPG_FORCING_NONE : f->dry_mode;
    p.dry_velocity_m_s = f->dry_velocity_m_s;
    if (p.dry_mode == FPG_FORCING_PER_PARTICLE) {
        if (!f->dry_velocity_per_slot) return FPG_ERR_INVALID_ARGUMENT;
        if ((st = upload_forcing(d, 0, f->dry_velocity_per_slot))) return st;
        p.dry_velocity_dev = d->d_forcing[0];
    }
    const bool wet_zero = f->wet_mode == FPG_FORCING_UNIFORM && f->wet_lambda_s_inv == 0.0f && f->wet_fraction == 0.0f;
    p.wet_mode = wet_zero ? FPG_FORCING_NONE : f->wet_mode;
    p.wet_lambda_s_inv = f->wet_lambda_s_inv;
    p.wet_fraction = f->wet_fraction;
    if (p.wet_mode == FPG_FORCING_PER_PARTICLE) {
        if (!f->wet_lambda_per_slot || !f->wet_fraction_per_slot) return FPG_ERR_INVALID_ARGUMENT;
        if ((st = upload_forcing(d, 1, f->wet_lambda_per_slot))) return st;
        if ((st = upload_forcing(d, 2, f->wet_fraction_per_slot))) return st;
        p.wet_lambda_dev = d->d_forcing[1];
        p.wet_fraction_dev = d->d_forcing[2];
    }
    p.wet_cells = f->wet_cells;

    // The reference dispatches `dispatch` slots (capacity, or the active
    // count with compaction); only [0, next_free) can hold particles.
    const size_t ref_dispatch = d->compaction ? d->active : d->capacity;
    d->particles->dispatch = d->next_free;
    uint32_t ignored[4];
    if (d->validation) {
        // the validation path (timeloop.rs:1128-1155): advection, Hanna
        // records, the Langevin update from the records, deposition, each a
        // pass of its own; the same bits as the fused kernel
        fpg_step_params pa = p;
        pa.stages = FPG_STAGE_ADVECT;
        st = fpg_step(d->ctx, d->particles, d->met, nullptr, &pa, nullptr, nullptr);
        const size_t n = d->particles->dispatch;
        if (st == FPG_OK)
            st = fpg_dispatch_hanna_params(d->ctx, d->particles, d->pbl, d->hanna_records, n, nullptr);
        if (st == FPG_OK)
            st = fpg_langevin_with_hanna(d->ctx, d->particles, d->hanna_records, n, p.turb_dt_seconds,
                                         p.rho_grad_over_rho, p.n_substeps, p.min_height_m, p.key, p.counter,
                                         ignored, nullptr);
        fpg_step_params pd = p;
        pd.stages = FPG_STAGE_DRY | FPG_STAGE_WET;
        if (st == FPG_OK) st = fpg_step(d->ctx, d->particles, nullptr, nullptr, &pd, nullptr, nullptr);
    } else {
        st = fpg_step(d->ctx, d->particles, d->met, d->pbl, &p, ignored, nullptr);
    }
    d->particles->dispatch = ref_dispatch;
    if (st != FPG_OK) return st;
    if (ref_dispatch > 0) {
        // gpu/langevin_fused.rs:229-233
        const uint64_t bpp = d->cfg.n_substeps <= 2u ? 1u : 2u;
        const uint64_t off = (uint64_t)ref_dispatch * bpp;
        const uint32_t lo = (uint32_t)off, hi = (uint32_t)(off >> 32);
        uint32_t c0 = d->counter[0] + lo;
        const uint32_t carry0 = c0 < d->counter[0];
        const uint32_t n1 = d->counter[1] + hi;
        const uint32_t carry1a = n1 < d->counter[1];
        const uint32_t c1 = n1 + carry0;
        const uint32_t carry1b = c1 < n1;
        const uint32_t c2 = d->counter[2] + (carry1a | carry1b);
        const uint32_t carry2 = c2 < d->counter[2];
        d->counter[0] = c0;
        d->counter[1] = c1;
        d->counter[2] = c2;
        d->counter[3] = d->counter[3] + carry2;
    }

    step_kernel_range.end();
    mark(d, 5);
    // compaction (timeloop.rs:1185-1197,1249-1262)
    if (d->compaction) {
        NvtxRange r("compaction");
        uint32_t act = 0;
        d->particles->dispatch = d->capacity;
        if ((st = fpg_compact(d->ctx, d->particles, d->compaction, &act, nullptr, nullptr))) return st;
        d->active = act;
        d->next_free = act;                       // reset_after_compaction (particles/mod.rs:600-605)
        d->particles->dispatch = act;
    }

    if (report) {
        report->step_index = d->step_index;
        report->simulation_time_seconds = d->t;
        report->interpolation_alpha = alpha;
        report->released_count = released;
        report->first_released_slot = first_slot;
        report->active_particle_count = d->active;
        std::memcpy(report->next_philox_counter, d->counter, sizeof(d->counter));
    }
    mark(d, 6);
    // the step is done: advance the clock before the timing read-back, so a
    // failed read leaves the driver consistent
    const uint64_t step_index = d->step_index;
    d->step_index += 1;
    d->t += d->direction > 0 ? d->cfg.timestep_seconds : -d->cfg.timestep_seconds;
    if (d->profile) {
        // StepTimingReport (timeloop.rs:398-467): device sections from the events
        const double host_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host_t0).count();
        FPG_CUDA(cudaEventSynchronize(d->marks[6]));
        double sec[6];
        for (int k = 0; k < 6; ++k) {
            float ms = 0.0f;
            FPG_CUDA(cudaEventElapsedTime(&ms, d->marks[k], d->marks[k + 1]));
            sec[k] = ms;
        }
        float total = 0.0f;
        FPG_CUDA(cudaEventElapsedTime(&total, d->marks[0], d->marks[6]));
        fpg_step_timing& t = d->last_timing;
        t.step_index = step_index;
        t.sort_ms = sec[0]; t.release_ms = sec[1]; t.met_bracket_ms = sec[2];
        t.pbl_ms = sec[3]; t.step_ms = sec[4]; t.compaction_ms = sec[5];
        t.gpu_total_ms = total;
        t.host_call_ms = host_ms;
        t.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host_t0).count();
        d->have_timing = true;
        if (d->print_profile)
            std::fprintf(stderr,
                         "[profile] step=%llu reorder=%.3fms release=%.3fms met_bracket=%.3fms pbl=%.3fms "
                         "step=%.3fms compaction=%.3fms gpu=%.3fms host_call=%.3fms total=%.3fms\n",
                         (unsigned long long)t.step_index, t.sort_ms, t.release_ms, t.met_bracket_ms, t.pbl_ms,
                         t.step_ms, t.compaction_ms, t.gpu_total_ms, t.host_call_ms, t.wall_ms);
    }
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_met_ring(fpg_forward* d, uint32_t n_slots) {
    if (!d || n_slots < 2) return FPG_ERR_INVALID_ARGUMENT;
    if (!d->ring.empty()) return d->ring.size() == n_slots ? FPG_OK : FPG_ERR_INVALID_ARGUMENT;
    const size_t nodes = d->met->nx * d->met->ny * d->met->nz, cells = d->met->nx * d->met->ny;
    cudaError_t e = cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking);
    d->ring.resize(n_slots);
    for (auto& slot : d->ring) {
        if (e == cudaSuccess) e = cudaMalloc(&slot.uvw, 3 * nodes * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&slot.surface, cells * sizeof(fpg_surface_cell));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.copied, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.released, cudaEventDisableTiming);
    }
    return e == cudaSuccess ? FPG_OK : cuda_status(e);
}

extern "C" fpg_status fpg_forward_prefetch_frame(fpg_forward* d, int64_t t, const float* u, const float* v,
                                                 const float* w, const fpg_surface_cell* surface) {
    if (!d || !u || !v || !w || !surface) return FPG_ERR_INVALID_ARGUMENT;
    if (d->ring.empty()) return FPG_ERR_NOT_READY;
    if (ring_find(d, t) >= 0) return FPG_OK;
    // victim: a free slot, else the least recently used outside the current bracket
    int victim = -1;
    for (size_t i = 0; i < d->ring.size(); ++i) {
        const fpg_forward::MetSlot& slot = d->ring[i];
        if (!slot.valid) { victim = (int)i; break; }
        if (d->have_bracket && (slot.time == d->bracket_t0 || slot.time == d->bracket_t1)) continue;
        if (victim < 0 || slot.last_use < d->ring[victim].last_use) victim = (int)i;
    }
    if (victim < 0) return FPG_ERR_STORE_FULL;
    fpg_forward::MetSlot& slot = d->ring[victim];
    const size_t nodes = d->met->nx * d->met->ny * d->met->nz, cells = d->met->nx * d->met->ny;
    cudaStream_t cs = d->copy_stream;
    FPG_CUDA(cudaStreamWaitEvent(cs, slot.released, 0));
    // host or device memory (the copy kind follows the pointer, unified addressing)
    FPG_CUDA(cudaMemcpyAsync(slot.uvw, u, nodes * sizeof(float), cudaMemcpyDefault, cs));
    FPG_CUDA(cudaMemcpyAsync(slot.uvw + nodes, v, nodes * sizeof(float), cudaMemcpyDefault, cs));
    FPG_CUDA(cudaMemcpyAsync(slot.uvw + 2 * nodes, w, nodes * sizeof(float), cudaMemcpyDefault, cs));
    FPG_CUDA(cudaMemcpyAsync(slot.surface, surface, cells * sizeof(fpg_surface_cell), cudaMemcpyDefault, cs));
    FPG_CUDA(cudaEventRecord(slot.copied, cs));
    slot.valid = true;
    slot.time = t;
    slot.last_use = ++d->tick;
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_met_ring_stats(const fpg_forward* d, uint64_t* hits, uint64_t* uploads) {
    if (!d) return FPG_ERR_INVALID_ARGUMENT;
    if (hits) *hits = d->ring_hits;
    if (uploads) *uploads = d->host_uploads;
    return FPG_OK;
}

extern "C" fpg_status fpg_forward_accumulate_grid(fpg_forward* d, fpg_grid* grid, uint32_t species, float scale,
                                                  const float* outheights, size_t n_oh) {
    if (!d || !grid) return FPG_ERR_INVALID_ARGUMENT;
    const size_t keep = d->particles->dispatch;
    d->particles->dispatch = d->next_free;
    const fpg_status st = fpg_grid_accumulate(d->ctx, d->particles, grid, species, scale, outheights, n_oh, nullptr);
    d->particles->dispatch = keep;
    return st;
}

// ============================================================================
// Backward (receptor) mode: BackwardTimeLoopDriver (timeloop.rs:1433-1909)
// ============================================================================

namespace fpg {
namespace {

struct RegionBox { double lon_min, lon_max, lat_min, lat_max, z_min, z_max; };

// collect_source_collections (timeloop.rs:1865-1894) in one pass: a particle
// is a hit of a region when its lon = xlon0 + (cell_x + pos_x) * dx, lat
// likewise and z lie inside the inclusive bounds (contains_particle,
// :187-197, in double).  Counts are warp-aggregated integer sums; masses are
// summed in double.  The loop runs in whole warps so every lane reaches the
// warp votes.
__global__ void __launch_bounds__(256) region_collect_kernel(const int32_t* __restrict__ cell_x,
                                                             const int32_t* __restrict__ cell_y,
                                                             const float* __restrict__ pos_x,
                                                             const float* __restrict__ pos_y,
                                                             const float* __restrict__ pos_z,
                                                             const uint32_t* __restrict__ flags,
                                                             const float* __restrict__ mass0, uint32_t n,
                                                             const RegionBox* __restrict__ regions,
                                                             uint32_t n_regions, fpg_grid_domain g,
                                                             unsigned long long* __restrict__ hits,
                                                             double* __restrict__ mass) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t p = base + threadIdx.x;
        const bool active = p < n && (flags[p] & 1u);
        double lon = 0.0, lat = 0.0, z = 0.0, m = 0.0;
        if (active) {
            lon = g.xlon0 + ((double)cell_x[p] + (double)pos_x[p]) * g.dx;
            lat = g.ylat0 + ((double)cell_y[p] + (double)pos_y[p]) * g.dy;
            z = (double)pos_z[p];
            m = (double)mass0[p];
        }
        for (uint32_t r = 0; r < n_regions; ++r) {
            const RegionBox b = regions[r];
            const bool in = active && lon >= b.lon_min && lon <= b.lon_max && lat >= b.lat_min &&
                            lat <= b.lat_max && z >= b.z_min && z <= b.z_max;
            const unsigned vote = __ballot_sync(0xffffffffu, in);
            if (vote == 0u) continue;
            double ms = in ? m : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ms += __shfl_xor_sync(0xffffffffu, ms, o);
            if (lane == 0u) {
                atomicAdd(hits + r, (unsigned long long)__popc(vote));
                atomicAdd(mass + r, ms);
            }
        }
    }
}

}  // namespace
}  // namespace fpg

struct fpg_backward {
    fpg_forward* f = nullptr;
    std::vector<RegionBox> regions;
    RegionBox* d_regions = nullptr;
    unsigned long long* d_hits = nullptr;
    double* d_mass = nullptr;
};

extern "C" void fpg_backward_config_default(fpg_backward_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->start_seconds = 1704067200;   // 20240101000000
    c->end_seconds = 1704067200;
    c->timestep_seconds = 1;
    c->clamp_time_bounds = 1;
    c->x_grid_per_meter = c->y_grid_per_meter = c->z_grid_per_meter = 1.0f;
    c->pbl_options = fpg_pbl_options{0.1f, 10.0f, 1.0f, 800.0f, 100.0f, 4500.0f};
    c->dry_reference_height_m = 15.0f;
    c->philox_key[0] = 0xDECAFBADu;
    c->philox_key[1] = 0x12345678u;
    c->n_substeps = 4;
    c->min_height_m = 0.01f;
}

extern "C" fpg_status fpg_backward_destroy(fpg_backward* b) {
    if (!b) return FPG_OK;
    fpg_forward_destroy(b->f);
    cudaFree(b->d_regions);
    cudaFree(b->d_hits);
    cudaFree(b->d_mass);
    delete b;
    return FPG_OK;
}

extern "C" fpg_status fpg_backward_create(fpg_ctx* ctx, const fpg_backward_config* cfg,
                                          const fpg_receptor_release* rec, size_t n_rec,
                                          const fpg_source_region* reg, size_t n_reg, const fpg_grid_domain* grid,
                                          size_t capacity, size_t nx, size_t ny, size_t nz, const float* heights,
                                          fpg_backward** out) {
    if (!ctx || !cfg || !grid || !out || (n_rec && !rec) || (n_reg && !reg)) return FPG_ERR_INVALID_ARGUMENT;
    // validate_backward_config (timeloop.rs:1974-2003), validate_receptor
    // (:2006-2046), validate_source_region (:2049-2073)
    if (cfg->start_seconds < cfg->end_seconds) return FPG_ERR_INVALID_BACKWARD_TIME_RANGE;
    if (cfg->timestep_seconds <= 0) return FPG_ERR_INVALID_TIME_STEP;
    if (!std::isfinite(cfg->dry_reference_height_m) || cfg->dry_reference_height_m <= 0.0f)
        return FPG_ERR_INVALID_REFERENCE_HEIGHT;
    if (n_rec == 0) return FPG_ERR_MISSING_RECEPTORS;
    for (size_t i = 0; i < n_rec; ++i) {
        const fpg_receptor_release& r = rec[i];
        if (!(r.lon >= -180.0 && r.lon <= 180.0) || !(r.lat >= -90.0 && r.lat <= 90.0) ||
            !std::isfinite(r.z_m) || r.z_m < 0.0 || r.particle_count == 0 || !std::isfinite(r.mass_kg) ||
            r.mass_kg <= 0.0)
            return FPG_ERR_INVALID_RECEPTOR;
    }
    for (size_t i = 0; i < n_reg; ++i)
        if (reg[i].lon_min > reg[i].lon_max || reg[i].lat_min > reg[i].lat_max || reg[i].z_min_m > reg[i].z_max_m)
            return FPG_ERR_INVALID_SOURCE_BOUNDS;
    // the driver over build_receptor_release_configs (timeloop.rs:1896-1917):
    // each receptor a point release of all its particles at the start time
    fpg_forward_config fc;
    fpg_forward_config_default(&fc);
    fc.start_seconds = cfg->start_seconds;
    fc.end_seconds = cfg->end_seconds;
    fc.timestep_seconds = cfg->timestep_seconds;
    fc.clamp_time_bounds = cfg->clamp_time_bounds;
    fc.x_grid_per_meter = cfg->x_grid_per_meter;
    fc.y_grid_per_meter = cfg->y_grid_per_meter;
    fc.z_grid_per_meter = cfg->z_grid_per_meter;
    fc.pbl_options = cfg->pbl_options;
    fc.dry_reference_height_m = cfg->dry_reference_height_m;
    std::memcpy(fc.philox_key, cfg->philox_key, sizeof(fc.philox_key));
    std::memcpy(fc.initial_philox_counter, cfg->initial_philox_counter, sizeof(fc.initial_philox_counter));
    fc.sort_interval_steps = 0;
    fc.use_compaction = 0;
    fc.n_substeps = cfg->n_substeps;
    fc.min_height_m = cfg->min_height_m;
    std::vector<fpg_release> rel(n_rec);
    for (size_t i = 0; i < n_rec; ++i) {
        fpg_release& r = rel[i];
        r.start_seconds = r.end_seconds = cfg->start_seconds;
        r.lon_min = r.lon_max = rec[i].lon;
        r.lat_min = r.lat_max = rec[i].lat;
        r.z_min = r.z_max = rec[i].z_m;
        r.mass_kg = rec[i].mass_kg;
        r.particle_count = rec[i].particle_count;
    }
    fpg_backward* b = new fpg_backward();
    fpg_status st = driver_create(ctx, &fc, rel.data(), n_rec, grid, capacity, nx, ny, nz, heights, -1, &b->f);
    if (st != FPG_OK) {
        delete b;
        return st;
    }
    for (size_t i = 0; i < n_reg; ++i)
        b->regions.push_back(RegionBox{reg[i].lon_min, reg[i].lon_max, reg[i].lat_min, reg[i].lat_max,
                                       reg[i].z_min_m, reg[i].z_max_m});
    const size_t nr = std::max<size_t>(n_reg, 1);
    cudaError_t e = cudaMalloc(&b->d_regions, nr * sizeof(RegionBox));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_hits, nr * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_mass, nr * sizeof(double));
    if (e == cudaSuccess && n_reg)
        e = cudaMemcpyAsync(b->d_regions, b->regions.data(), n_reg * sizeof(RegionBox), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        fpg_backward_destroy(b);
        return cuda_status(e);
    }
    *out = b;
    return FPG_OK;
}

extern "C" int32_t fpg_backward_has_remaining_steps(const fpg_backward* b) {
    return b ? fpg_forward_has_remaining_steps(b->f) : 0;
}
extern "C" int64_t fpg_backward_current_time(const fpg_backward* b) { return b ? fpg_forward_current_time(b->f) : 0; }
extern "C" fpg_particles* fpg_backward_particles(fpg_backward* b) { return b ? b->f->particles : nullptr; }

extern "C" fpg_status fpg_backward_set_validation_mode(fpg_backward* b, int32_t on) {
    return b ? fpg_forward_set_validation_mode(b->f, on) : FPG_ERR_INVALID_ARGUMENT;
}

extern "C" fpg_status fpg_backward_run_timestep(fpg_backward* b, const fpg_met_bracket* met, const fpg_forcing* f,
                                                fpg_step_report* report, fpg_source_collection* out) {
    if (!b) return FPG_ERR_INVALID_ARGUMENT;
    fpg_status st = fpg_forward_run_timestep(b->f, met, f, report);
    if (st != FPG_OK) return st;
    fpg_forward* d = b->f;
    cudaStream_t s = d->ctx->stream;
    const size_t nr = b->regions.size();
    if (nr) {
        FPG_CUDA(cudaMemsetAsync(b->d_hits, 0, nr * sizeof(unsigned long long), s));
        FPG_CUDA(cudaMemsetAsync(b->d_mass, 0, nr * sizeof(double), s));
        const uint32_t n = (uint32_t)d->next_free;
        if (n) {
            fpg_particles* P = d->particles;
            const uint32_t blocks = std::min<uint32_t>((n + 255u) / 256u, (uint32_t)d->ctx->sm_count * 8u);
            region_collect_kernel<<<blocks, 256, 0, s>>>(
                (const int32_t*)P->field[FPG_FIELD_CELL_X], (const int32_t*)P->field[FPG_FIELD_CELL_Y],
                (const float*)P->field[FPG_FIELD_POS_X], (const float*)P->field[FPG_FIELD_POS_Y],
                (const float*)P->field[FPG_FIELD_POS_Z], (const uint32_t*)P->field[FPG_FIELD_FLAGS],
                (const float*)P->field[FPG_FIELD_MASS0], n, b->d_regions, (uint32_t)nr, d->domain, b->d_hits,
                b->d_mass);
            d->ctx->count();
            FPG_CHECK_LAUNCH();
        }
    }
    std::vector<unsigned long long> hits(nr);
    std::vector<double> mass(nr);
    if (nr) {
        FPG_CUDA(cudaMemcpyAsync(hits.data(), b->d_hits, nr * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        FPG_CUDA(cudaMemcpyAsync(mass.data(), b->d_mass, nr * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    // the reference waits for the device every backward step (timeloop.rs:1798)
    FPG_CUDA(cudaStreamSynchronize(s));
    if (out)
        for (size_t r = 0; r < nr; ++r) {
            out[r].hit_count = hits[r];
            out[r].total_mass_kg = (float)mass[r];
            out[r].pad = 0.0f;
            out[r].total_mass_kg_f64 = mass[r];
        }
    return FPG_OK;
}
