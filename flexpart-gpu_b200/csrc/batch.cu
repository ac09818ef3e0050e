// batch.cu — many independent release scenarios stepped as one population.
//
// Each scenario reproduces one plain forward run (ForwardTimeLoopDriver with
// a single release, capacity = its particle count, its own Philox key and
// counter chain; src/simulation/timeloop.rs:915-1316): release lattice and
// slots (release/mod.rs:156-275), Philox block index = slot within the
// scenario, counter advanced by capacity * blocks per step
// (gpu/langevin_fused.rs:229-233).  All scenarios share one met frame ring
// and one clock.  Scenario s owns the 256-aligned slot segment
// [offset_s, offset_s + capacity_s) of one structure-of-arrays population;
// tile t (256 slots) belongs to exactly one scenario.
//
// One step is a fixed kernel sequence that reads its per-step values
// (clock, alpha, bracket, release ranges, counters) from device memory, so
// it is captured once into a CUDA graph and replayed:
//   batch_advance   clock -> bracket + alpha; per-scenario release ranges
//   batch_pack      repack the bracket from the ring when it changed
//   batch_pbl       surface lerp + PBL per cell (+ wet forcing on a change)
//   batch_release   new particles of every scenario (lattice in f64)
//   batch_step      persistent: CTAs pull 256-slot tiles from a work queue
//                   and run the fused per-particle step (step_core.cuh)
//   batch_grid_*    per-scenario grids at output steps
//   batch_end       counters += capacity * blocks; clock += dt
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <algorithm>
#include <vector>

#include "../../include/fpg_driver.h"
#include "batch_core.cuh"
#include "fpg_internal.h"
#include "grid_core.cuh"

namespace fpg {

size_t particles_block_bytes(size_t capacity);

// the plain fused step (step.cu), launched once per scenario by the sequential path
__global__ void __launch_bounds__(256, 5) fused_step_kernel(StepArgs a);

namespace {


__global__ void batch_advance_kernel(BatchState* st, ScenDev* sc, BatchConst c) {
    const int64_t t = st->t;
    if (threadIdx.x == 0) {
        // bracket holding t; at a frame time stay in the bracket ending there
        int64_t k = (t - c.start) / c.frame_seconds;
        if (t - c.start == k * c.frame_seconds && k > 0) k -= 1;
        const int32_t fa = (int32_t)(k % c.n_frames), fb = (int32_t)((k + 1) % c.n_frames);
        const int64_t ta = c.start + k * c.frame_seconds;
        st->changed = !st->have_bracket || fa != st->fa || fb != st->fb || ta != st->ta;
        st->fa = fa;
        st->fb = fb;
        st->ta = ta;
        st->have_bracket = 1;
        // interpolation_alpha (timeloop.rs:2117-2119)
        st->alpha = (float)((double)(t - ta) / (double)c.frame_seconds);
        st->work = 0;
    }
    for (uint32_t s = threadIdx.x; s < c.n_scen; s += blockDim.x) {
        ScenDev& d = sc[s];
        const uint32_t lo = d.released;
        uint32_t hi = target_emitted(d.start, d.end, d.count, t, lo);
        if (hi < lo) hi = lo;
        d.rel_lo = lo;
        d.rel_hi = hi;
        d.released = hi;
    }
}

__global__ void __launch_bounds__(256) batch_pack_kernel(const BatchState* st, const float4* __restrict__ ring,
                                                         uint32_t nodes, float4* __restrict__ bracket) {
    if (!st->changed) return;
    const float4* f0 = ring + (size_t)st->fa * nodes;
    const float4* f1 = ring + (size_t)st->fb * nodes;
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < nodes; n += gridDim.x * blockDim.x) {
        st_node(bracket, n, f0[n], f1[n]);
    }
}

__global__ void __launch_bounds__(256) batch_pbl_kernel(const BatchState* st, const fpg_surface_cell* __restrict__ sring,
                                                        const float* __restrict__ precip, fpg_pbl_options o,
                                                        uint32_t ncell, float* f0, float* f1, float* f2, float* f3,
                                                        float* f4, float* f5, float* f6, float4* packed,
                                                        CellHanna* hanna, int wet_on,
                                                        float wa, float wb, float2* wet) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    pbl_cell(sring + (size_t)st->fa * ncell, sring + (size_t)st->fb * ncell, st->alpha, o, c, f0, f1, f2, f3, f4, f5,
             f6, packed, hanna);
    if (wet_on && st->changed) wet[c] = wet_cell_forcing(precip[(size_t)st->fa * ncell + c], 0.0f, 1.0f, wa, wb);
}

// ReleaseManager::inject_for_time + geo_to_grid + to_relative
// (release/mod.rs:103-146, coords/mod.rs:92-114,169-178) on the device, in
// the same f64 arithmetic as the host release manager.
__global__ void __launch_bounds__(256) batch_release_kernel(BatchState* st, const ScenDev* __restrict__ sc,
                                                            BatchConst c, PopFields F) {
    const ScenDev& d = sc[blockIdx.y];
    const int32_t now = (int32_t)st->t;
    for (uint32_t k = d.rel_lo + blockIdx.x * blockDim.x + threadIdx.x; k < d.rel_hi; k += gridDim.x * blockDim.x) {
        const uint64_t idx = k;
        const uint64_t ix = idx % d.lat_nx, iy = (idx / d.lat_nx) % d.lat_nx, iz = (idx / d.lat_nxy) % d.lat_nz;
        const double fx = ((double)ix + 0.5) / (double)d.lat_nx;
        const double fy = ((double)iy + 0.5) / (double)d.lat_nx;
        const double fz = ((double)iz + 0.5) / (double)d.lat_nz;
        const double lon = d.lon_min + fx * (d.lon_max - d.lon_min);
        const double lat = d.lat_min + fy * (d.lat_max - d.lat_min);
        const double z = d.z_min + fz * (d.z_max - d.z_min);
        const double x = (lon - c.xlon0) / c.dx;
        const double y = (lat - c.ylat0) / c.dy;
        if (!(x >= 0.0 && x < (double)(c.gnx - 1) && y >= 0.0 && y < (double)(c.gny - 1))) {
            atomicOr(&st->error, 1);
            continue;
        }
        const double fxf = floor(x), fyf = floor(y);
        const uint32_t p = d.offset + k;
        F.f[FPG_FIELD_CELL_X][p] = (uint32_t)(int32_t)fxf;
        F.f[FPG_FIELD_CELL_Y][p] = (uint32_t)(int32_t)fyf;
        F.f[FPG_FIELD_POS_X][p] = __float_as_uint((float)(x - fxf));
        F.f[FPG_FIELD_POS_Y][p] = __float_as_uint((float)(y - fyf));
        F.f[FPG_FIELD_POS_Z][p] = __float_as_uint((float)z);
        F.f[FPG_FIELD_FLAGS][p] = FPG_FLAG_ACTIVE;
        F.f[FPG_FIELD_MASS0][p] = __float_as_uint(d.mass_per_particle);
        F.f[FPG_FIELD_TIME][p] = (uint32_t)now;
        F.f[FPG_FIELD_TIME_MEM][p] = (uint32_t)now;
        // every other field of a fresh slot is zero (the population starts zeroed)
    }
}

// One work item is a chunk of BLOCK * PPT consecutive slots of one scenario
// (x: scenario, y: first slot within the scenario).  CTAs stay resident and
// pull items from a device counter until none is left, so small and large
// scenarios share the machine without a per-scenario launch.
template <int BLOCK, int MINB, int PPT>
__global__ void __launch_bounds__(BLOCK, MINB) batch_step_kernel(StepArgs a, BatchState* st,
                                                                 const ScenDev* __restrict__ sc,
                                                                 const uint2* __restrict__ items, uint32_t n_items) {
    extern __shared__ float s_levels[];
    __shared__ uint32_t s_item;
    const Levels lv = stage_levels(a, s_levels);
    const float alpha = st->alpha;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(&st->work, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= n_items) break;
        const uint2 w = items[it];
        const ScenDev& d = sc[w.x];
        const uint32_t released = d.released;
#pragma unroll 1
        for (int j = 0; j < PPT; ++j) {
            const uint32_t local = w.y + (uint32_t)(j * BLOCK) + threadIdx.x;
            if (local < released)
                particle_step(a, lv, d.offset + local, local, alpha, d.counter, d.key0, d.key1);
        }
    }
}

// The same pass with one CTA per work item of BLOCK slots, launched over all
// items (particles_per_thread 0 in the tuning records): no work counter and
// no barrier, the level arrays read from global memory, and the hardware's
// block scheduler spreading the items of small and large scenarios.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) batch_step_flat_kernel(StepArgs a, BatchState* st,
                                                                      const ScenDev* __restrict__ sc,
                                                                      const uint2* __restrict__ items,
                                                                      uint32_t n_items) {
    if (blockIdx.x >= n_items) return;
    const uint2 w = items[blockIdx.x];
    const ScenDev& d = sc[w.x];
    const uint32_t local = w.y + threadIdx.x;
    if (local < d.released)
        particle_step(a, global_levels(a), d.offset + local, local, st->alpha, d.counter, d.key0, d.key1);
}

// The launch shapes the particle pass is compiled for; the tuner picks one,
// and the first is the default.  ppt 0: batch_step_flat_kernel, one CTA per
// item of `block` slots.
struct StepVariant {
    uint32_t block, minb, ppt;
    void (*kernel)(StepArgs, BatchState*, const ScenDev*, const uint2*, uint32_t);
};

const StepVariant kVariants[] = {
    {128, 12, 0, batch_step_flat_kernel<128, 12>},
    {256, 4, 1, batch_step_kernel<256, 4, 1>}, {256, 4, 2, batch_step_kernel<256, 4, 2>},
    {256, 3, 1, batch_step_kernel<256, 3, 1>}, {256, 2, 1, batch_step_kernel<256, 2, 1>},
    {128, 8, 1, batch_step_kernel<128, 8, 1>}, {128, 8, 2, batch_step_kernel<128, 8, 2>},
    {512, 2, 1, batch_step_kernel<512, 2, 1>}, {256, 5, 1, batch_step_kernel<256, 5, 1>},
    {256, 5, 0, batch_step_flat_kernel<256, 5>}, {128, 10, 0, batch_step_flat_kernel<128, 10>},
};
static_assert(sizeof(kVariants) / sizeof(kVariants[0]) == kNumVariants, "launch shape table");

struct GridConst {
    uint32_t nx, ny, nz, cells;
    int meters, sorted;
    float scale;
    uint32_t every;
    float h[FPG_MAX_LEVELS];
    float lower[kSortedLevels - 1];     // level_sorted's table when `sorted`
};

__global__ void __launch_bounds__(256) batch_grid_clear_kernel(const BatchState* st, uint32_t every, uint32_t* counts,
                                                               uint32_t* mass, size_t total) {
    if (every == 0 || (st->step + 1u) % every != 0u) return;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        counts[i] = 0u;
        mass[i] = 0u;
    }
}

// concentration_gridding.wgsl:323-345 per scenario.  Each CTA bins a
// contiguous range of tiles (a tile is 256 slots of one scenario); the key of
// a particle is its index in the scenario-major grid, so one CTA table holds
// the cells of every scenario its tiles touch.  Runs of equal keys in a warp
// are summed by the segmented scan, the run ends add to the table, and the
// table goes to the grids once per cell per CTA (grid_core.cuh).
__global__ void __launch_bounds__(256) batch_grid_kernel(const BatchState* st, const ScenDev* __restrict__ sc,
                                                         const uint32_t* __restrict__ tile_scen, PopFields F,
                                                         GridConst g, uint32_t n_tiles, uint32_t tiles_per_cta,
                                                         uint32_t* counts, uint32_t* mass) {
    if (g.every == 0 || (st->step + 1u) % g.every != 0u) return;
    __shared__ float s_h[FPG_MAX_LEVELS];
    __shared__ uint32_t t_key[kTable], t_cnt[kTable], t_mass[kTable];
    if (!g.sorted)
        for (uint32_t i = threadIdx.x; i < g.nz; i += blockDim.x) s_h[i] = g.h[i];
    for (uint32_t i = threadIdx.x; i < kTable; i += blockDim.x) {
        t_key[i] = kEmpty;
        t_cnt[i] = 0u;
        t_mass[i] = 0u;
    }
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t t0 = blockIdx.x * tiles_per_cta;
    const uint32_t t1 = min(t0 + tiles_per_cta, n_tiles);
    for (uint32_t tile = t0; tile < t1; ++tile) {                       // uniform across the CTA
        const uint32_t s = tile_scen[tile];
        const ScenDev& d = sc[s];
        const uint32_t local = (tile - d.first_tile) * TILE + threadIdx.x;
        const uint32_t p = d.offset + local;
        uint32_t key = kEmpty, q = 0u;
        if (local < d.released && (F.f[FPG_FIELD_FLAGS][p] & 1u)) {
            const int32_t cx = (int32_t)F.f[FPG_FIELD_CELL_X][p], cy = (int32_t)F.f[FPG_FIELD_CELL_Y][p];
            const uint32_t ix = (uint32_t)min(max(cx, 0), (int)g.nx - 1);
            const uint32_t iy = (uint32_t)min(max(cy, 0), (int)g.ny - 1);
            const float z = __uint_as_float(F.f[FPG_FIELD_POS_Z][p]);
            const uint32_t iz = g.sorted ? level_sorted(z, g.lower, g.nz) : level_of(z, s_h, g.nz, g.meters);
            key = s * g.cells + (ix * g.ny + iy) * g.nz + iz;
            q = quantize(fmaxf(__uint_as_float(F.f[FPG_FIELD_MASS0][p]), 0.0f), g.scale);
        }
        warp_runs_add(key, q, lane, t_key, t_cnt, t_mass, counts, mass);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kTable; i += blockDim.x) {
        const uint32_t k = t_key[i];
        if (k != kEmpty) {
            atomicAdd(counts + k, t_cnt[i]);
            atomicAdd(mass + k, t_mass[i]);
        }
    }
}

__global__ void batch_end_kernel(BatchState* st, ScenDev* sc, BatchConst c) {
    for (uint32_t s = threadIdx.x; s < c.n_scen; s += blockDim.x)
        sc[s].counter = counter_add64(sc[s].counter, (uint64_t)sc[s].capacity * c.bpp);
    if (threadIdx.x == 0) {
        st->t += c.dt;
        st->step += 1u;
    }
}

}  // namespace

StepArgs make_step_args(fpg_batch* b) {
    fpg_particles* P = b->pop;
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.cell_x = (int32_t*)P->field[FPG_FIELD_CELL_X];
    a.cell_y = (int32_t*)P->field[FPG_FIELD_CELL_Y];
    a.pos_x = (float*)P->field[FPG_FIELD_POS_X];
    a.pos_y = (float*)P->field[FPG_FIELD_POS_Y];
    a.pos_z = (float*)P->field[FPG_FIELD_POS_Z];
    a.flags = (const uint32_t*)P->field[FPG_FIELD_FLAGS];
    for (int k = 0; k < 4; ++k) a.mass[k] = (float*)P->field[FPG_FIELD_MASS0 + k];
    a.vel_u = (float*)P->field[FPG_FIELD_VEL_U];
    a.vel_v = (float*)P->field[FPG_FIELD_VEL_V];
    a.vel_w = (float*)P->field[FPG_FIELD_VEL_W];
    a.turb_u = (float*)P->field[FPG_FIELD_TURB_U];
    a.turb_v = (float*)P->field[FPG_FIELD_TURB_V];
    a.turb_w = (float*)P->field[FPG_FIELD_TURB_W];
    a.cbt = (int32_t*)P->field[FPG_FIELD_CBT];
    a.n = (uint32_t)P->capacity;
    a.n_species = 1;                                  // each release fills species 0 only
    const fpg_batch_config& c = b->cfg;
    a.stages = FPG_STAGE_ADVECT | FPG_STAGE_TURBULENCE;
    a.bracket = b->met->bracket;
    a.heights = b->met->heights_dev;
    a.nx = (uint32_t)b->met->nx; a.ny = (uint32_t)b->met->ny; a.nz = (uint32_t)b->met->nz;
    a.has_heights = b->met->heights_set && b->met->heights[b->met->nz - 1] > 0.0f;
    a.level_mode = level_mode(b->met);
    a.level_table = b->met->level_table_dev;
    a.level_inv_w = b->met->level_inv_w;
    a.dt = (float)c.timestep_seconds;
    a.xs = c.x_grid_per_meter; a.ys = c.y_grid_per_meter; a.zs = c.z_grid_per_meter;
    a.hcell = b->pbl->hanna;
    a.pnx = (uint32_t)b->pbl->nx; a.pny = (uint32_t)b->pbl->ny;
    a.tdt = (float)c.timestep_seconds;
    a.rho = c.rho_grad_over_rho;
    a.zmin = c.min_height_m;
    a.n_sub = c.n_substeps;
    a.href = fmaxf(c.dry_reference_height_m, 0.1f);
    a.dry_mode = c.dry_velocity_m_s != 0.0f ? FPG_FORCING_UNIFORM : FPG_FORCING_NONE;
    if (a.dry_mode) a.stages |= FPG_STAGE_DRY;
    a.dry_v = c.dry_velocity_m_s;
    a.wet_mode = c.wet_from_precipitation ? FPG_FORCING_PER_CELL : FPG_FORCING_NONE;
    if (a.wet_mode) {
        a.stages |= FPG_STAGE_WET;
        a.wet_cells = b->wet->lf;
        a.wnx = (uint32_t)b->wet->nx; a.wny = (uint32_t)b->wet->ny;
    }
    return a;
}

BatchConst make_const(const fpg_batch* b) {
    BatchConst c;
    c.start = b->cfg.start_seconds;
    c.frame_seconds = b->cfg.frame_seconds;
    c.dt = b->cfg.timestep_seconds;
    c.n_frames = b->cfg.n_frames;
    c.n_scen = (uint32_t)b->scen.size();
    c.n_tiles = b->n_tiles;
    c.bpp = b->cfg.n_substeps <= 2u ? 1u : 2u;
    c.xlon0 = b->cfg.release_grid.xlon0; c.ylat0 = b->cfg.release_grid.ylat0;
    c.dx = b->cfg.release_grid.dx; c.dy = b->cfg.release_grid.dy;
    c.gnx = b->cfg.release_grid.nx; c.gny = b->cfg.release_grid.ny;
    return c;
}

GridConst make_grid_const(const fpg_batch* b) {
    GridConst g;
    std::memset(&g, 0, sizeof(g));
    g.nx = b->cfg.out_nx; g.ny = b->cfg.out_ny; g.nz = b->cfg.out_nz;
    g.cells = g.nx * g.ny * g.nz;
    for (uint32_t k = 0; k < g.nz; ++k) g.h[k] = b->outheights[k];
    g.meters = g.nz > 0 && g.h[g.nz - 1] > 0.0f;
    g.sorted = sorted_levels(g.h, g.nz, g.lower);
    g.scale = 1.0e6f;
    g.every = b->cfg.output_every_steps;
    return g;
}

PopFields pop_fields(fpg_batch* b) {
    PopFields F;
    for (int f = 0; f < FPG_FIELD_COUNT; ++f) F.f[f] = static_cast<uint32_t*>(b->pop->field[f]);
    return F;
}

// The per-step kernels before and after the particle pass (shared by the
// batched and sequential paths).
void enqueue_pre(fpg_batch* b, cudaStream_t s) {
    const BatchConst c = make_const(b);
    const uint32_t nodes = (uint32_t)(b->met->nx * b->met->ny * b->met->nz);
    const uint32_t cells = (uint32_t)(b->pbl->nx * b->pbl->ny);
    batch_advance_kernel<<<1, 256, 0, s>>>(b->st, b->sc, c);
    batch_pack_kernel<<<b->ctx->sm_count * 4, 256, 0, s>>>(b->st, b->ring, nodes, b->met->bracket);
    batch_pbl_kernel<<<(cells + 255) / 256, 256, 0, s>>>(
        b->st, b->sring, b->pring, b->cfg.pbl_options, cells, b->pbl->field[0], b->pbl->field[1], b->pbl->field[2],
        b->pbl->field[3], b->pbl->field[4], b->pbl->field[5], b->pbl->field[6], b->pbl->packed, b->pbl->hanna,
        b->cfg.wet_from_precipitation, b->cfg.wet_gas_a, b->cfg.wet_gas_b, b->wet ? b->wet->lf : nullptr);
    batch_release_kernel<<<dim3(16, (unsigned)b->scen.size()), 256, 0, s>>>(b->st, b->sc, c, pop_fields(b));
    b->ctx->count(4);
}

void enqueue_post(fpg_batch* b, cudaStream_t s) {
    const BatchConst c = make_const(b);
    const GridConst g = make_grid_const(b);
    const size_t total = (size_t)g.cells * b->scen.size();
    if (g.every && g.cells && b->n_tiles) {
        batch_grid_clear_kernel<<<b->ctx->sm_count * 4, 256, 0, s>>>(b->st, g.every, b->grid_counts, b->grid_mass,
                                                                     total);
        // 8 resident CTAs per SM, each over a contiguous range of tiles
        const uint32_t ctas = std::max<uint32_t>(1u, std::min<uint32_t>(b->n_tiles, (uint32_t)b->ctx->sm_count * 8u));
        const uint32_t per = (b->n_tiles + ctas - 1u) / ctas;
        const uint32_t blocks = std::max<uint32_t>(1u, (b->n_tiles + per - 1u) / per);
        batch_grid_kernel<<<blocks, 256, 0, s>>>(b->st, b->sc, b->tile_scen, pop_fields(b), g, b->n_tiles, per,
                                                 b->grid_counts, b->grid_mass);
        b->ctx->count(2);
    }
    if (b->inv) enqueue_inverse_sample(b, s);
    batch_end_kernel<<<1, 256, 0, s>>>(b->st, b->sc, c);
    b->ctx->count(1);
}

void enqueue_end(fpg_batch* b, cudaStream_t s) {
    batch_end_kernel<<<1, 256, 0, s>>>(b->st, b->sc, make_const(b));
    b->ctx->count(1);
}

void enqueue_step_kernel(fpg_batch* b, cudaStream_t s) {
    const StepVariant& v = kVariants[b->variant];
    const StepArgs a = make_step_args(b);
    if (v.ppt == 0) {
        v.kernel<<<std::max(b->n_items, 1u), v.block, 0, s>>>(a, b->st, b->sc, b->items, b->n_items);
    } else {
        const uint32_t grid = (uint32_t)b->ctx->sm_count * std::max(b->resident[b->variant], 1u);
        v.kernel<<<grid, v.block, level_smem_bytes(b->met), s>>>(a, b->st, b->sc, b->items, b->n_items);
    }
    b->ctx->count(1);
}

void enqueue_batched_step(fpg_batch* b, cudaStream_t s) {
    enqueue_pre(b, s);
    enqueue_step_kernel(b, s);
    enqueue_post(b, s);
}

// Work items of shape `v`: every scenario cut into chunks of block * ppt slots.
fpg_status build_items(fpg_batch* b, uint32_t v) {
    const uint32_t chunk = kVariants[v].block * std::max(kVariants[v].ppt, 1u);
    std::vector<uint2> items;
    for (size_t s = 0; s < b->scen.size(); ++s)
        for (uint32_t l = 0; l < b->scen[s].capacity; l += chunk) items.push_back(make_uint2((uint32_t)s, l));
    if (items.size() > b->items_cap) {
        cudaFree(b->items);
        b->items = nullptr;
        b->items_cap = 0;
        FPG_CUDA(cudaMalloc(&b->items, items.size() * sizeof(uint2)));
        b->items_cap = items.size();
    }
    FPG_CUDA(cudaMemcpyAsync(b->items, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                             b->ctx->stream));
    FPG_CUDA(cudaStreamSynchronize(b->ctx->stream));
    b->n_items = (uint32_t)items.size();
    b->variant = v;
    // a captured graph holds the old shape
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    return FPG_OK;
}

__global__ void __launch_bounds__(256) batch_pack_forced_kernel(const BatchState* st, const float4* __restrict__ ring,
                                                                uint32_t nodes, float4* __restrict__ bracket) {
    const float4* f0 = ring + (size_t)st->fa * nodes;
    const float4* f1 = ring + (size_t)st->fb * nodes;
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < nodes; n += gridDim.x * blockDim.x) {
        st_node(bracket, n, f0[n], f1[n]);
    }
}

void enqueue_pack_forced(fpg_batch* b, const BatchState* st, cudaStream_t s) {
    const uint32_t nodes = (uint32_t)(b->met->nx * b->met->ny * b->met->nz);
    batch_pack_forced_kernel<<<b->ctx->sm_count * 4, 256, 0, s>>>(st, b->ring, nodes, b->met->bracket);
    b->ctx->count(1);
}

fpg_status batch_reset(fpg_batch* b) {
    cudaStream_t s = b->ctx->stream;
    FPG_CUDA(cudaMemsetAsync(b->pop->block, 0, particles_block_bytes(b->capacity), s));
    BatchState s0;
    std::memset(&s0, 0, sizeof(s0));
    s0.t = b->cfg.start_seconds;
    FPG_CUDA(cudaMemcpyAsync(b->st, &s0, sizeof(s0), cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(b->sc, b->scen.data(), b->scen.size() * sizeof(ScenDev), cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaStreamSynchronize(s));
    b->steps_done = 0;
    b->t_h = b->cfg.start_seconds;
    for (size_t k = 0; k < b->scen.size(); ++k) {
        b->released_h[k] = 0;
        b->counter_h[k] = b->scen[k].counter;
    }
    return FPG_OK;
}

fpg_status ensure_graph(fpg_batch* b) {
    if (b->exec) return FPG_OK;
    cudaStream_t s = b->ctx->stream;
    FPG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = b->ctx->launches.load();
    enqueue_batched_step(b, s);
    // capture launches nothing: take the count back, keep it per replay
    b->graph_launches = b->ctx->launches.load() - before;
    b->ctx->launches.fetch_sub(b->graph_launches);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) return cuda_status(e);
    b->graph = g;
    FPG_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    return FPG_OK;
}

// ReleaseError::OutOfGridDomain (release/mod.rs:41) of scenario d, checked at
// the lattice's extreme points (lon, lat grow monotonically with the lattice
// index, so every other point lies between them).
fpg_status check_release_grid(const ScenDev& d, const fpg_grid_domain& g) {
    const uint64_t ix_hi = std::min<uint64_t>(d.lat_nx - 1, d.count - 1);
    const uint64_t iy_hi = std::min<uint64_t>(d.lat_nx - 1, (d.count - 1) / d.lat_nx);
    for (int e = 0; e < 4; ++e) {
        const uint64_t ix = (e & 1) ? ix_hi : 0, iy = (e & 2) ? iy_hi : 0;
        const double lon = d.lon_min + (((double)ix + 0.5) / (double)d.lat_nx) * (d.lon_max - d.lon_min);
        const double lat = d.lat_min + (((double)iy + 0.5) / (double)d.lat_nx) * (d.lat_max - d.lat_min);
        const double x = (lon - g.xlon0) / g.dx;
        const double y = (lat - g.ylat0) / g.dy;
        if (!(x >= 0.0 && x < (double)(g.nx - 1) && y >= 0.0 && y < (double)(g.ny - 1))) return FPG_ERR_OUT_OF_GRID;
    }
    return FPG_OK;
}

}  // namespace fpg

using namespace fpg;

extern "C" fpg_status fpg_batch_destroy(fpg_batch* b) {
    if (!b) return FPG_OK;
    cudaStreamSynchronize(b->ctx->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    fpg_particles_destroy(b->pop);
    fpg_met_destroy(b->met);
    fpg_pbl_destroy(b->pbl);
    fpg_cellfield_destroy(b->wet);
    cudaFree(b->ring); cudaFree(b->sring); cudaFree(b->pring); cudaFree(b->staging);
    cudaFree(b->st); cudaFree(b->sc); cudaFree(b->tile_scen); cudaFree(b->items); cudaFree(b->grid_counts); cudaFree(b->grid_mass);
    delete b;
    return FPG_OK;
}

extern "C" fpg_status fpg_batch_create(fpg_ctx* ctx, const fpg_batch_config* cfg, const fpg_batch_scenario* scen,
                                       size_t n_scen, size_t nx, size_t ny, size_t nz, const float* heights,
                                       fpg_batch** out) {
    if (!ctx || !cfg || !out || !scen || n_scen == 0 || n_scen > 65535) return FPG_ERR_INVALID_ARGUMENT;
    if (cfg->start_seconds > cfg->end_seconds) return FPG_ERR_INVALID_TIME_RANGE;
    if (cfg->timestep_seconds <= 0 || cfg->frame_seconds <= 0 || cfg->n_frames == 0) return FPG_ERR_INVALID_TIME_STEP;
    if (cfg->output_every_steps && (cfg->out_nx == 0 || cfg->out_ny == 0 || cfg->out_nz == 0)) return FPG_ERR_ZERO_SHAPE;
    if (cfg->out_nz > FPG_MAX_LEVELS) return FPG_ERR_TOO_MANY_LEVELS;
    fpg_batch* b = new fpg_batch();
    b->ctx = ctx;
    b->cfg = *cfg;
    if (cfg->outheights && cfg->out_nz) b->outheights.assign(cfg->outheights, cfg->outheights + cfg->out_nz);
    else b->outheights.assign(cfg->out_nz, 0.0f);
    b->cfg.outheights = nullptr;
    size_t offset = 0;
    for (size_t s = 0; s < n_scen; ++s) {
        const fpg_release& r = scen[s].release;
        if (r.lon_min > r.lon_max || r.lat_min > r.lat_max || r.z_min > r.z_max) { delete b; return FPG_ERR_INVALID_BOUNDS; }
        if (r.particle_count == 0 || r.particle_count >= (1ull << 32) || r.end_seconds - r.start_seconds >= (1ll << 32)) {
            delete b;
            return FPG_ERR_VALUE_TOO_LARGE;
        }
        ScenDev d;
        std::memset(&d, 0, sizeof(d));
        d.offset = (uint32_t)offset;
        d.capacity = (uint32_t)r.particle_count;
        d.first_tile = (uint32_t)(offset / TILE);
        d.n_tiles = (uint32_t)((r.particle_count + TILE - 1) / TILE);
        d.key0 = scen[s].key[0]; d.key1 = scen[s].key[1];
        d.counter = u32x4{scen[s].counter[0], scen[s].counter[1], scen[s].counter[2], scen[s].counter[3]};
        d.mass_per_particle = (float)(r.mass_kg / (double)r.particle_count);
        d.start = r.start_seconds; d.end = r.end_seconds;
        d.lon_min = r.lon_min; d.lon_max = r.lon_max; d.lat_min = r.lat_min; d.lat_max = r.lat_max;
        d.z_min = r.z_min; d.z_max = r.z_max;
        d.count = r.particle_count;
        // the lattice size of ReleaseBounds::sample_stratified (release/mod.rs:257-260), computed on the host
        double c = std::ceil(std::cbrt((double)r.particle_count));
        if (c < 1.0) c = 1.0;
        d.lat_nx = (uint64_t)c;
        d.lat_nxy = d.lat_nx * d.lat_nx > 0 ? d.lat_nx * d.lat_nx : 1;
        d.lat_nz = (r.particle_count + d.lat_nxy - 1) / d.lat_nxy;
        if (d.lat_nz < 1) d.lat_nz = 1;
        if (check_release_grid(d, cfg->release_grid) != FPG_OK) {
            delete b;
            return FPG_ERR_OUT_OF_GRID;
        }
        b->scen.push_back(d);
        for (uint32_t t = 0; t < d.n_tiles; ++t) b->tile_scen_h.push_back((uint32_t)s);
        offset += (size_t)d.n_tiles * TILE;
    }
    if (offset >= (size_t)UINT32_MAX) { delete b; return FPG_ERR_VALUE_TOO_LARGE; }
    b->capacity = offset;
    b->n_tiles = (uint32_t)b->tile_scen_h.size();
    b->total_steps = (uint64_t)((cfg->end_seconds - cfg->start_seconds) / cfg->timestep_seconds) + 1;
    b->released_h.assign(n_scen, 0);
    for (const ScenDev& d : b->scen) b->counter_h.push_back(d.counter);
    b->t_h = cfg->start_seconds;

    fpg_status st = fpg_particles_create(ctx, b->capacity, &b->pop);
    if (st == FPG_OK) st = fpg_met_create(ctx, nx, ny, nz, &b->met);
    if (st == FPG_OK && heights) st = fpg_met_set_level_heights(b->met, heights, nz);
    if (st == FPG_OK) st = fpg_pbl_create(ctx, nx, ny, &b->pbl);
    if (st == FPG_OK && cfg->wet_from_precipitation) st = fpg_cellfield_create(ctx, nx, ny, &b->wet);
    if (st != FPG_OK) { fpg_batch_destroy(b); return st; }
    b->met->uploaded[0] = b->met->uploaded[1] = true;   // the graph packs the bracket on the device
    b->pbl->ready = true;
    if (b->wet) b->wet->ready = true;
    const size_t nodes = nx * ny * nz, cells = nx * ny;
    const size_t grid_total = (size_t)cfg->out_nx * cfg->out_ny * cfg->out_nz * n_scen;
    cudaError_t e = cudaMalloc(&b->ring, nodes * cfg->n_frames * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&b->sring, cells * cfg->n_frames * sizeof(fpg_surface_cell));
    if (e == cudaSuccess) e = cudaMalloc(&b->pring, cells * cfg->n_frames * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->staging, nodes * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&b->st, sizeof(BatchState));
    if (e == cudaSuccess) e = cudaMalloc(&b->sc, n_scen * sizeof(ScenDev));
    if (e == cudaSuccess) e = cudaMalloc(&b->tile_scen, b->n_tiles * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->grid_counts, (grid_total ? grid_total : 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->grid_mass, (grid_total ? grid_total : 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->pring, 0, cells * cfg->n_frames * sizeof(float), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->grid_counts, 0, (grid_total ? grid_total : 1) * 4, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->grid_mass, 0, (grid_total ? grid_total : 1) * 4, ctx->stream);
    BatchState s0;
    std::memset(&s0, 0, sizeof(s0));
    s0.t = cfg->start_seconds;
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->st, &s0, sizeof(s0), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->sc, b->scen.data(), n_scen * sizeof(ScenDev), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->tile_scen, b->tile_scen_h.data(), b->n_tiles * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { fpg_batch_destroy(b); return cuda_status(e); }
    for (uint32_t v = 0; v < kNumVariants; ++v) {
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kVariants[v].kernel, (int)kVariants[v].block,
                                                          nz * sizeof(float) + FPG_LEVEL_BUCKETS);
        if (e != cudaSuccess) { fpg_batch_destroy(b); return cuda_status(e); }
        b->resident[v] = (uint32_t)std::max(per_sm, 1);
    }
    st = build_items(b, 0);
    if (st != FPG_OK) { fpg_batch_destroy(b); return st; }
    *out = b;
    return FPG_OK;
}

namespace fpg {
__global__ void __launch_bounds__(256) batch_pack_ring_kernel(const float* __restrict__ u, const float* __restrict__ v,
                                                              const float* __restrict__ w, uint32_t nodes, float4* out) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nodes) out[n] = make_float4(u[n], v[n], w[n], 0.0f);
}
}  // namespace fpg

extern "C" fpg_status fpg_batch_upload_frame(fpg_batch* b, uint32_t k, const float* u, const float* v, const float* w,
                                             const fpg_surface_cell* surface, const float* precip) {
    if (!b || !u || !v || !w || !surface || k >= b->cfg.n_frames) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = b->ctx->stream;
    const size_t nodes = b->met->nx * b->met->ny * b->met->nz, cells = b->met->nx * b->met->ny;
    FPG_CUDA(cudaMemcpyAsync(b->staging, u, nodes * 4, cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(b->staging + nodes, v, nodes * 4, cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(b->staging + 2 * nodes, w, nodes * 4, cudaMemcpyHostToDevice, s));
    batch_pack_ring_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(b->staging, b->staging + nodes,
                                                                          b->staging + 2 * nodes, (uint32_t)nodes,
                                                                          b->ring + k * nodes);
    b->ctx->count();
    FPG_CHECK_LAUNCH();
    FPG_CUDA(cudaMemcpyAsync(b->sring + k * cells, surface, cells * sizeof(fpg_surface_cell), cudaMemcpyHostToDevice, s));
    if (precip) FPG_CUDA(cudaMemcpyAsync(b->pring + k * cells, precip, cells * 4, cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaStreamSynchronize(s));
    return FPG_OK;
}

extern "C" fpg_status fpg_batch_run(fpg_batch* b, uint32_t n_steps, int32_t use_graph) {
    if (!b) return FPG_ERR_INVALID_ARGUMENT;
    if (b->steps_done >= b->total_steps) return FPG_ERR_SIMULATION_COMPLETE;
    const uint64_t n = std::min<uint64_t>(n_steps, b->total_steps - b->steps_done);
    cudaStream_t s = b->ctx->stream;
    if (use_graph) {
        const fpg_status st = ensure_graph(b);
        if (st != FPG_OK) return st;
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (use_graph) {
            FPG_CUDA(cudaGraphLaunch(b->exec, s));
            b->ctx->count(b->graph_launches);
        } else {
            enqueue_batched_step(b, s);
            FPG_CHECK_LAUNCH();
        }
    }
    // keep the host mirror (used by the sequential path) in step
    const uint32_t bpp = b->cfg.n_substeps <= 2u ? 1u : 2u;
    for (uint64_t i = 0; i < n; ++i) {
        for (size_t k = 0; k < b->scen.size(); ++k) {
            const ScenDev& d = b->scen[k];
            uint32_t hi = target_emitted(d.start, d.end, d.count, b->t_h, b->released_h[k]);
            if (hi > b->released_h[k]) b->released_h[k] = hi;
            b->counter_h[k] = counter_add64(b->counter_h[k], (uint64_t)d.capacity * bpp);
        }
        b->t_h += b->cfg.timestep_seconds;
    }
    b->steps_done += n;
    return FPG_OK;
}

extern "C" fpg_status fpg_batch_run_sequential(fpg_batch* b, uint32_t n_steps) {
    if (!b) return FPG_ERR_INVALID_ARGUMENT;
    if (b->steps_done >= b->total_steps) return FPG_ERR_SIMULATION_COMPLETE;
    const uint64_t n = std::min<uint64_t>(n_steps, b->total_steps - b->steps_done);
    cudaStream_t s = b->ctx->stream;
    const uint32_t bpp = b->cfg.n_substeps <= 2u ? 1u : 2u;
    StepArgs base = make_step_args(b);
    // alpha of the step comes from the host clock (same formula as the device)
    for (uint64_t i = 0; i < n; ++i) {
        enqueue_pre(b, s);
        int64_t k = (b->t_h - b->cfg.start_seconds) / b->cfg.frame_seconds;
        if (b->t_h - b->cfg.start_seconds == k * b->cfg.frame_seconds && k > 0) k -= 1;
        const int64_t ta = b->cfg.start_seconds + k * b->cfg.frame_seconds;
        const float alpha = (float)((double)(b->t_h - ta) / (double)b->cfg.frame_seconds);
        for (size_t sidx = 0; sidx < b->scen.size(); ++sidx) {
            const ScenDev& d = b->scen[sidx];
            uint32_t hi = target_emitted(d.start, d.end, d.count, b->t_h, b->released_h[sidx]);
            if (hi > b->released_h[sidx]) b->released_h[sidx] = hi;
            const uint32_t released = b->released_h[sidx];
            const u32x4 counter = b->counter_h[sidx];
            // the counter advances every step, released particles or not (as the driver's)
            b->counter_h[sidx] = counter_add64(counter, (uint64_t)d.capacity * bpp);
            if (released == 0) continue;
            // one plain launch of the fused step over this scenario's segment
            StepArgs a = base;
            const uint32_t o = d.offset;
            a.cell_x += o; a.cell_y += o; a.pos_x += o; a.pos_y += o; a.pos_z += o; a.flags += o;
            for (int m = 0; m < 4; ++m) a.mass[m] += o;
            a.vel_u += o; a.vel_v += o; a.vel_w += o; a.turb_u += o; a.turb_v += o; a.turb_w += o; a.cbt += o;
            a.n = released;
            a.alpha = alpha;
            a.key0 = d.key0; a.key1 = d.key1;
            a.counter = counter;
            fused_step_kernel<<<(released + 255) / 256, 256, 0, s>>>(a);
            b->ctx->count();
        }
        enqueue_post(b, s);
        FPG_CHECK_LAUNCH();
        b->t_h += b->cfg.timestep_seconds;
    }
    b->steps_done += n;
    return FPG_OK;
}

extern "C" uint64_t fpg_batch_steps_done(const fpg_batch* b) { return b ? b->steps_done : 0; }

extern "C" fpg_status fpg_batch_scenario_slots(const fpg_batch* b, size_t s, size_t* first, size_t* count) {
    if (!b || s >= b->scen.size() || !first || !count) return FPG_ERR_INVALID_ARGUMENT;
    *first = b->scen[s].offset;
    *count = b->scen[s].capacity;
    return FPG_OK;
}

extern "C" fpg_particles* fpg_batch_particles(fpg_batch* b) { return b ? b->pop : nullptr; }

extern "C" fpg_status fpg_batch_download_grids(fpg_batch* b, uint32_t* counts, uint32_t* mass) {
    if (!b) return FPG_ERR_INVALID_ARGUMENT;
    const size_t total = (size_t)b->cfg.out_nx * b->cfg.out_ny * b->cfg.out_nz * b->scen.size();
    cudaStream_t s = b->ctx->stream;
    if (counts) FPG_CUDA(cudaMemcpyAsync(counts, b->grid_counts, total * 4, cudaMemcpyDeviceToHost, s));
    if (mass) FPG_CUDA(cudaMemcpyAsync(mass, b->grid_mass, total * 4, cudaMemcpyDeviceToHost, s));
    FPG_CUDA(cudaStreamSynchronize(s));
    return FPG_OK;
}

extern "C" fpg_status fpg_batch_errors(fpg_batch* b, int32_t* flags) {
    if (!b || !flags) return FPG_ERR_INVALID_ARGUMENT;
    BatchState h;
    FPG_CUDA(cudaMemcpyAsync(&h, b->st, sizeof(h), cudaMemcpyDeviceToHost, b->ctx->stream));
    FPG_CUDA(cudaStreamSynchronize(b->ctx->stream));
    *flags = h.error;
    return FPG_OK;
}

// ---- launch-shape tuner ------------------------------------------------------

extern "C" uint32_t fpg_batch_tuning_candidates(fpg_batch_tuning* out, uint32_t max) {
    for (uint32_t v = 0; out && v < kNumVariants && v < max; ++v)
        out[v] = fpg_batch_tuning{kVariants[v].block, kVariants[v].minb, kVariants[v].ppt, 0.0f};
    return kNumVariants;
}

static int find_variant(const fpg_batch_tuning* t) {
    for (uint32_t v = 0; v < kNumVariants; ++v)
        if (kVariants[v].block == t->block_threads && kVariants[v].minb == t->min_blocks_per_sm &&
            kVariants[v].ppt == t->particles_per_thread)
            return (int)v;
    return -1;
}

extern "C" fpg_status fpg_batch_set_tuning(fpg_batch* b, const fpg_batch_tuning* t) {
    if (!b || !t) return FPG_ERR_INVALID_ARGUMENT;
    const int v = find_variant(t);
    if (v < 0) return FPG_ERR_INVALID_ARGUMENT;
    b->tuned_ms = t->step_ms;
    return build_items(b, (uint32_t)v);
}

extern "C" fpg_status fpg_batch_get_tuning(const fpg_batch* b, fpg_batch_tuning* t) {
    if (!b || !t) return FPG_ERR_INVALID_ARGUMENT;
    const StepVariant& v = kVariants[b->variant];
    *t = fpg_batch_tuning{v.block, v.minb, v.ppt, b->tuned_ms};
    return FPG_OK;
}

// Times the particle pass of the next step under every compiled launch
// shape, each from the same snapshot of the live state (population, clock,
// release and counter state), restores the snapshot and keeps the fastest
// shape.  Each particle's arithmetic does not depend on the launch shape, so
// the choice changes speed only, never results.
extern "C" fpg_status fpg_batch_autotune(fpg_batch* b, uint32_t reps, fpg_batch_tuning* results, uint32_t max_results,
                                         fpg_batch_tuning* best) {
    if (!b) return FPG_ERR_INVALID_ARGUMENT;
    if (b->steps_done >= b->total_steps) return FPG_ERR_SIMULATION_COMPLETE;
    if (reps == 0) reps = 1;
    cudaStream_t s = b->ctx->stream;
    const size_t pop_bytes = particles_block_bytes(b->capacity);
    const size_t sc_bytes = b->scen.size() * sizeof(ScenDev);
    void* snap = nullptr;
    BatchState* st_snap = nullptr;
    ScenDev* sc_snap = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    fpg_status status = FPG_OK;
    uint32_t best_v = b->variant;
    float best_ms = 0.0f;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMalloc(&snap, pop_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&st_snap, sizeof(BatchState));
    if (e == cudaSuccess) e = cudaMalloc(&sc_snap, sc_bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(snap, b->pop->block, pop_bytes, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st_snap, b->st, sizeof(BatchState), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sc_snap, b->sc, sc_bytes, cudaMemcpyDeviceToDevice, s);
    auto restore = [&]() {
        cudaError_t r = cudaMemcpyAsync(b->pop->block, snap, pop_bytes, cudaMemcpyDeviceToDevice, s);
        if (r == cudaSuccess) r = cudaMemcpyAsync(b->st, st_snap, sizeof(BatchState), cudaMemcpyDeviceToDevice, s);
        if (r == cudaSuccess) r = cudaMemcpyAsync(b->sc, sc_snap, sc_bytes, cudaMemcpyDeviceToDevice, s);
        return r;
    };
    for (uint32_t v = 0; e == cudaSuccess && status == FPG_OK && v < kNumVariants; ++v) {
        status = build_items(b, v);
        float tmin = 0.0f;
        for (uint32_t r = 0; status == FPG_OK && e == cudaSuccess && r < reps; ++r) {
            e = restore();
            if (e != cudaSuccess) break;
            enqueue_pre(b, s);
            e = cudaEventRecord(e0, s);
            if (e != cudaSuccess) break;
            enqueue_step_kernel(b, s);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && (r == 0 || ms < tmin)) tmin = ms;
        }
        if (e != cudaSuccess || status != FPG_OK) break;
        if (results && v < max_results)
            results[v] = fpg_batch_tuning{kVariants[v].block, kVariants[v].minb, kVariants[v].ppt, tmin};
        if (v == 0 || tmin < best_ms) { best_ms = tmin; best_v = v; }
    }
    if (e == cudaSuccess) e = restore();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(snap); cudaFree(st_snap); cudaFree(sc_snap);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_status(e);
    if (status != FPG_OK) return status;
    status = build_items(b, best_v);
    b->tuned_ms = best_ms;
    if (best) fpg_batch_get_tuning(b, best);
    return status;
}
