// grid.cu — concentration gridding (concentration_gridding.wgsl:284-345,
// host side src/gpu/gridding.rs:255-420).
//
// Each active particle adds 1 to its cell's count and u32(mass*scale+0.5) to
// its cell's scaled mass.  Both grids are u32 sums, so the result is the same
// whatever order the additions happen in.  Plumes put ~1e5 particles in a
// cell, so one global atomic per particle (or per warp) serialises on the
// hot cells: a warp first merges the particles that share a cell, a CTA
// merges its warps' sums in a shared-memory table over one contiguous chunk
// of slots, and the grid receives one pair of atomics per distinct cell per
// CTA.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "fpg_internal.h"
#include "grid_core.cuh"

namespace fpg {

// The output heights: all of them for the scan, and when they are sorted and
// at most kSortedLevels (`sorted`), the first nz - 1 padded with +inf for the
// branch-free count (level_sorted).
struct LevelTable {
    float h[FPG_MAX_LEVELS];
    float lower[kSortedLevels - 1];
    int sorted;
};

struct GridArgs {
    const int32_t* cell_x; const int32_t* cell_y; const float* pos_z; const uint32_t* flags; const float* mass;
    uint32_t n, nx, ny, nz;
    float mass_scale;
    int meters;  // outheights[nz-1] > 0
};

__device__ __forceinline__ uint32_t cell_of(const GridArgs& a, const float* h, uint32_t p) {
    const int32_t cx = a.cell_x[p], cy = a.cell_y[p];
    const uint32_t ix = (uint32_t)min(max(cx, 0), (int)a.nx - 1);
    const uint32_t iy = (uint32_t)min(max(cy, 0), (int)a.ny - 1);
    const uint32_t iz = level_of(a.pos_z[p], h, a.nz, a.meters);
    return (ix * a.ny + iy) * a.nz + iz;
}

// Each thread bins two adjacent slots per pass (one 64-bit load per field).
constexpr uint32_t kSlotsPerThread = 2;

struct SlotPair {
    uint2 f, cx, cy, z, m;      // flags, cell_x, cell_y, pos_z, mass (bits)
};

__device__ __forceinline__ void load_pair(const GridArgs& a, uint64_t p, uint64_t end, SlotPair& s) {
    s.f = make_uint2(0u, 0u);
    if (p + 1u < end) {
        s.f = *reinterpret_cast<const uint2*>(a.flags + p);
        s.cx = *reinterpret_cast<const uint2*>(a.cell_x + p);
        s.cy = *reinterpret_cast<const uint2*>(a.cell_y + p);
        s.z = *reinterpret_cast<const uint2*>(a.pos_z + p);
        s.m = *reinterpret_cast<const uint2*>(a.mass + p);
    } else if (p < end) {
        s.f.x = a.flags[p];
        s.cx.x = (uint32_t)a.cell_x[p];
        s.cy.x = (uint32_t)a.cell_y[p];
        s.z.x = __float_as_uint(a.pos_z[p]);
        s.m.x = __float_as_uint(a.mass[p]);
    }
}

// The cell and the scaled mass of one slot (kEmpty and 0 when inactive).
__device__ __forceinline__ void slot_cell(const GridArgs& a, const LevelTable& lt, const float* s_h, uint32_t f,
                                          uint32_t cx, uint32_t cy, uint32_t zb, uint32_t mb, uint32_t& key,
                                          uint32_t& q) {
    key = kEmpty;
    q = 0u;
    if (f & 1u) {
        const uint32_t ix = (uint32_t)min(max((int32_t)cx, 0), (int)a.nx - 1);
        const uint32_t iy = (uint32_t)min(max((int32_t)cy, 0), (int)a.ny - 1);
        const float z = __uint_as_float(zb);
        const uint32_t iz = lt.sorted ? level_sorted(z, lt.lower, a.nz) : level_of(z, s_h, a.nz, a.meters);
        key = (ix * a.ny + iy) * a.nz + iz;
        q = quantize(fmaxf(__uint_as_float(mb), 0.0f), a.mass_scale);
    }
}

// Each CTA bins one contiguous chunk of slots.  The fields of the next pass
// are loaded before the current pass's warp sums and table updates, so a
// thread always has a pass of loads in flight.  A warp sums the runs of equal
// cells of its 32 even slots, then of its 32 odd ones (the reorder keeps
// neighbouring slots in one cell, so both stay long).  All sums are u32, so
// the grid does not depend on the order of the additions.
__global__ void __launch_bounds__(256) grid_kernel(GridArgs a, LevelTable lt, uint32_t chunk,
                                                   uint32_t* __restrict__ counts, uint32_t* __restrict__ mass) {
    __shared__ float s_h[FPG_MAX_LEVELS];
    __shared__ uint32_t t_key[kTable], t_cnt[kTable], t_mass[kTable];
    if (!lt.sorted)
        for (uint32_t i = threadIdx.x; i < a.nz; i += blockDim.x) s_h[i] = lt.h[i];
    for (uint32_t i = threadIdx.x; i < kTable; i += blockDim.x) {
        t_key[i] = kEmpty;
        t_cnt[i] = 0u;
        t_mass[i] = 0u;
    }
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t begin = (uint64_t)blockIdx.x * chunk;    // chunk: a multiple of the pass, so begin is even
    const uint64_t end = min(begin + chunk, (uint64_t)a.n);
    const uint64_t pass = (uint64_t)kSlotsPerThread * blockDim.x;
    const uint64_t mine = (uint64_t)kSlotsPerThread * threadIdx.x;
    SlotPair cur;
    load_pair(a, begin + mine, end, cur);
    __syncthreads();
    for (uint64_t base = begin; base < end; base += pass) {      // uniform across the CTA
        uint32_t k0, q0, k1, q1;
        slot_cell(a, lt, s_h, cur.f.x, cur.cx.x, cur.cy.x, cur.z.x, cur.m.x, k0, q0);
        slot_cell(a, lt, s_h, cur.f.y, cur.cx.y, cur.cy.y, cur.z.y, cur.m.y, k1, q1);
        if (base + pass < end) load_pair(a, base + pass + mine, end, cur);
        warp_runs_add(k0, q0, lane, t_key, t_cnt, t_mass, counts, mass);      // the even slots' runs
        warp_runs_add(k1, q1, lane, t_key, t_cnt, t_mass, counts, mass);      // the odd slots'
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

__global__ void __launch_bounds__(256) cell_index_kernel(GridArgs a, LevelTable lt, uint32_t* __restrict__ out) {
    __shared__ float s_h[FPG_MAX_LEVELS];
    for (uint32_t i = threadIdx.x; i < a.nz; i += blockDim.x) s_h[i] = lt.h[i];
    __syncthreads();
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    out[p] = (a.flags[p] & 1u) ? cell_of(a, s_h, p) : 0xffffffffu;
}

static fpg_status prepare(const fpg_particles* P, const fpg_grid* g, uint32_t species, float scale,
                          const float* oh, size_t n_oh, GridArgs& a, LevelTable& lt) {
    if (g->nx == 0 || g->ny == 0 || g->nz == 0) return FPG_ERR_ZERO_SHAPE;
    if (species >= FPG_MAX_SPECIES) return FPG_ERR_INVALID_SPECIES;            // gridding.rs:262
    if (!std::isfinite(scale) || scale <= 0.0f) return FPG_ERR_INVALID_MASS_SCALE;  // gridding.rs:268
    if (oh && n_oh != g->nz) return FPG_ERR_LENGTH_MISMATCH;
    if (P->dispatch > (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    std::memset(&lt, 0, sizeof(lt));
    if (oh) std::memcpy(lt.h, oh, g->nz * sizeof(float));
    lt.sorted = sorted_levels(lt.h, (uint32_t)g->nz, lt.lower);
    a.cell_x = (const int32_t*)P->field[FPG_FIELD_CELL_X];
    a.cell_y = (const int32_t*)P->field[FPG_FIELD_CELL_Y];
    a.pos_z = (const float*)P->field[FPG_FIELD_POS_Z];
    a.flags = (const uint32_t*)P->field[FPG_FIELD_FLAGS];
    a.mass = (const float*)P->field[FPG_FIELD_MASS0 + species];
    a.n = (uint32_t)P->dispatch;
    a.nx = (uint32_t)g->nx; a.ny = (uint32_t)g->ny; a.nz = (uint32_t)g->nz;
    a.mass_scale = scale;
    a.meters = lt.h[g->nz - 1] > 0.0f;
    return FPG_OK;
}

}  // namespace fpg

using namespace fpg;

extern "C" fpg_status fpg_grid_create(fpg_ctx* ctx, size_t nx, size_t ny, size_t nz, fpg_grid** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (nx == 0 || ny == 0 || nz == 0) return FPG_ERR_ZERO_SHAPE;
    if (nz > FPG_MAX_LEVELS) return FPG_ERR_TOO_MANY_LEVELS;
    if (nx * ny * nz >= (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_grid* g = new fpg_grid();
    g->ctx = ctx; g->nx = nx; g->ny = ny; g->nz = nz;
    const size_t cells = nx * ny * nz;
    cudaError_t e = cudaMalloc(&g->counts, cells * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&g->mass, cells * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(g->counts, 0, cells * sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(g->mass, 0, cells * sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->produced, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->copied, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        fpg_grid_destroy(g);
        return cuda_status(e);
    }
    g->last_stream = ctx->stream;
    *out = g;
    return FPG_OK;
}

extern "C" fpg_status fpg_grid_destroy(fpg_grid* g) {
    if (!g) return FPG_OK;
    if (g->copy_pending) cudaEventSynchronize(g->copied);
    cudaFree(g->counts);
    cudaFree(g->mass);
    if (g->produced) cudaEventDestroy(g->produced);
    if (g->copied) cudaEventDestroy(g->copied);
    delete g;
    return FPG_OK;
}

extern "C" fpg_status fpg_grid_download_async(fpg_grid* g, uint32_t* counts, uint32_t* mass_scaled, void* stream) {
    if (!g) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = g->ctx->pick(stream);
    const size_t cells = g->nx * g->ny * g->nz;
    if (s != g->last_stream) {
        FPG_CUDA(cudaEventRecord(g->produced, g->last_stream));
        FPG_CUDA(cudaStreamWaitEvent(s, g->produced, 0));
    }
    if (counts) FPG_CUDA(cudaMemcpyAsync(counts, g->counts, cells * 4, cudaMemcpyDeviceToHost, s));
    if (mass_scaled) FPG_CUDA(cudaMemcpyAsync(mass_scaled, g->mass, cells * 4, cudaMemcpyDeviceToHost, s));
    FPG_CUDA(cudaEventRecord(g->copied, s));
    g->copy_pending = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_grid_accumulate(fpg_ctx* ctx, const fpg_particles* P, fpg_grid* g, uint32_t species,
                                          float mass_scale, const float* outheights, size_t n_oh, void* stream) {
    if (!ctx || !P || !g) return FPG_ERR_INVALID_ARGUMENT;
    GridArgs a;
    LevelTable lt;
    fpg_status st = prepare(P, g, species, mass_scale, outheights, n_oh, a, lt);
    if (st != FPG_OK) return st;
    cudaStream_t s = ctx->pick(stream);
    const size_t cells = g->nx * g->ny * g->nz;
    if (g->copy_pending) {                  // an fpg_grid_download_async still reading the grid
        FPG_CUDA(cudaStreamWaitEvent(s, g->copied, 0));
        g->copy_pending = false;
    }
    g->last_stream = s;
    FPG_CUDA(cudaMemsetAsync(g->counts, 0, cells * sizeof(uint32_t), s));   // outputs.clear (gridding.rs:282)
    FPG_CUDA(cudaMemsetAsync(g->mass, 0, cells * sizeof(uint32_t), s));
    g->mass_scale = mass_scale;
    if (a.n == 0) return FPG_OK;
    // 8 resident CTAs per SM, one contiguous chunk each
    const uint32_t pass = 256u * kSlotsPerThread;
    const uint32_t tiles = (uint32_t)(((uint64_t)a.n + pass - 1u) / pass);
    const uint32_t ctas = std::min<uint32_t>(tiles, (uint32_t)ctx->sm_count * 8u);
    const uint32_t chunk = ((tiles + ctas - 1u) / ctas) * pass;
    const uint32_t blocks = (uint32_t)(((uint64_t)a.n + chunk - 1u) / chunk);
    grid_kernel<<<blocks, 256, 0, s>>>(a, lt, chunk, g->counts, g->mass);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}

extern "C" fpg_status fpg_grid_cell_indices(fpg_ctx* ctx, const fpg_particles* P, const fpg_grid* g,
                                            const float* outheights, size_t n_oh, uint32_t* out_dev, void* stream) {
    if (!ctx || !P || !g || !out_dev) return FPG_ERR_INVALID_ARGUMENT;
    GridArgs a;
    LevelTable lt;
    fpg_status st = prepare(P, g, 0, 1.0f, outheights, n_oh, a, lt);
    if (st != FPG_OK) return st;
    if (a.n == 0) return FPG_OK;
    cell_index_kernel<<<(a.n + 255) / 256, 256, 0, ctx->pick(stream)>>>(a, lt, out_dev);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}

extern "C" fpg_status fpg_grid_download(fpg_grid* g, uint32_t* counts, uint32_t* mass_scaled, float* mass_kg,
                                        void* stream) {
    if (!g) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = g->ctx->pick(stream);
    const size_t cells = g->nx * g->ny * g->nz;
    if (counts) FPG_CUDA(cudaMemcpyAsync(counts, g->counts, cells * 4, cudaMemcpyDeviceToHost, s));
    uint32_t* ms = mass_scaled;
    uint32_t* tmp = nullptr;
    if (!ms && mass_kg) {
        tmp = new uint32_t[cells];
        ms = tmp;
    }
    cudaError_t e = cudaSuccess;
    if (ms) e = cudaMemcpyAsync(ms, g->mass, cells * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && mass_kg) {
        // download_output (gridding.rs:210-213): (value as f32) / mass_scale
        for (size_t i = 0; i < cells; ++i) mass_kg[i] = (float)ms[i] / g->mass_scale;
    }
    delete[] tmp;
    return e == cudaSuccess ? FPG_OK : cuda_status(e);
}

extern "C" uint32_t* fpg_grid_counts_device(fpg_grid* g) { return g ? g->counts : nullptr; }
extern "C" uint32_t* fpg_grid_mass_device(fpg_grid* g) { return g ? g->mass : nullptr; }
