// sort.cu — reorder particles by met cell.
//
// The reference can reorder its particle store on the host by a Morton key
// of the quantised position every few steps (ParticleStore::sort_spatially,
// src/particles/mod.rs:649-699, applied by apply_spatial_sort_if_enabled,
// src/simulation/timeloop.rs:1414-1430) so that neighbouring slots sample
// neighbouring met.  Here the key is the 3-D met cell the particle sits in,
// ((ix*ny)+iy)*nz+iz with ix, iy, iz the lower corner indices the trilinear
// sample of the fused step uses, so a warp's 32 particles mostly share their
// 8 corner nodes (broadcast gathers) and their PBL cell (one stability
// regime, no divergence).  Inactive slots get key 0xFFFFFFFF and move to the
// end, as the reference's INACTIVE_MORTON_KEY does (particles/mod.rs:27);
// on the device that key is nx*ny*nz (one past the last cell) so the radix
// sort only runs over the bits the cell count needs.
//
// Steps: key kernel -> stable LSD radix sort of (key, slot) pairs (CUB,
// header-only, compiled into this library) -> gather of all FPG_FIELD_COUNT
// arrays into a second structure-of-arrays block, which is swapped in.
// Philox streams follow the slot, as in the reference after its sort.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include "fpg_internal.h"
#include "physics.cuh"

struct fpg_sorter {
    fpg_ctx* ctx = nullptr;
    size_t capacity = 0;
    uint32_t* keys[2] = {};
    uint32_t* vals[2] = {};
    void* temp = nullptr;
    size_t temp_bytes = 0;
    void* block = nullptr;
};

namespace fpg {

void particles_swap_block(fpg_particles* p, void** other_block);
size_t particles_block_bytes(size_t capacity);
void particles_assign_fields(void* block, size_t capacity, void** field);

struct KeyArgs {
    const int32_t* cell_x; const int32_t* cell_y; const float* pos_x; const float* pos_y; const float* pos_z;
    const uint32_t* flags;
    const float* heights;
    uint32_t n, nx, ny, nz;
    int has_heights, monotonic;
};

// Same lower-corner arithmetic as the fused step (axis_bracket and
// meters_to_level, advection_dual_wind.wgsl:94-138).
__device__ __forceinline__ uint32_t lower_index(float coord, uint32_t n) {
    return (uint32_t)floorf(clampf(coord, 0.0f, (float)(n - 1u)));
}

__device__ __forceinline__ float level_of_height(const float* h, uint32_t nz, int has, int mono, float z) {
    if (!has) return z;
    const float h0 = h[0];
    if (z <= h0) return h0 > 0.0f ? z / h0 : 0.0f;
    uint32_t k;
    if (mono) {
        uint32_t lo = 1u, hi = nz;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (z <= h[mid]) hi = mid; else lo = mid + 1u;
        }
        k = lo;
    } else {
        k = nz;
        for (uint32_t i = 1u; i < nz; ++i) if (z <= h[i]) { k = i; break; }
    }
    if (k >= nz) return (float)(nz - 1u);
    const float hprev = h[k - 1u];
    const float denom = h[k] - hprev;
    if (denom > 0.0f) return (float)(k - 1u) + (z - hprev) / denom;
    return (float)(k - 1u);
}

__global__ void __launch_bounds__(256) cell_key_kernel(KeyArgs a, uint32_t* __restrict__ keys,
                                                       uint32_t* __restrict__ vals) {
    extern __shared__ float s_h[];
    for (uint32_t i = threadIdx.x; i < a.nz; i += blockDim.x) s_h[i] = a.heights[i];
    __syncthreads();
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    uint32_t key = a.nx * a.ny * a.nz;
    if (a.flags[p] & FLAG_ACTIVE) {
        const uint32_t ix = lower_index((float)a.cell_x[p] + a.pos_x[p], a.nx);
        const uint32_t iy = lower_index((float)a.cell_y[p] + a.pos_y[p], a.ny);
        const uint32_t iz = lower_index(level_of_height(s_h, a.nz, a.has_heights, a.monotonic, a.pos_z[p]), a.nz);
        key = (ix * a.ny + iy) * a.nz + iz;
    }
    keys[p] = key;
    vals[p] = p;
}

struct SortFields { uint32_t* f[FPG_FIELD_COUNT]; };

// dst[f][i] = src[f][perm[i]] for i < n, dst[f][i] = src[f][i] above.
__global__ void __launch_bounds__(256) permute_kernel(SortFields src, SortFields dst, const uint32_t* __restrict__ perm,
                                                      uint32_t n, uint32_t capacity) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= capacity) return;
    const uint32_t s = i < n ? perm[i] : i;
#pragma unroll
    for (int f = 0; f < FPG_FIELD_COUNT; ++f) dst.f[f][i] = src.f[f][s];
}

// Bits needed for keys 0..cells (cells itself is the inactive key).
static int key_bits(size_t cells) {
    int b = 1;
    while (b < 32 && ((size_t)1 << b) <= cells) ++b;
    return b;
}

}  // namespace fpg

using namespace fpg;

extern "C" fpg_status fpg_sorter_create(fpg_ctx* ctx, size_t capacity, fpg_sorter** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (capacity > (size_t)INT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_sorter* s = new fpg_sorter();
    s->ctx = ctx;
    s->capacity = capacity;
    const size_t n = capacity > 0 ? capacity : 1;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMalloc(&s->keys[k], n * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMalloc(&s->vals[k], n * sizeof(uint32_t));
    }
    if (e == cudaSuccess) {
        cub::DoubleBuffer<uint32_t> kb(s->keys[0], s->keys[1]), vb(s->vals[0], s->vals[1]);
        e = cub::DeviceRadixSort::SortPairs(nullptr, s->temp_bytes, kb, vb, (int)n, 0, 32, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaMalloc(&s->temp, s->temp_bytes > 0 ? s->temp_bytes : 1);
    if (e == cudaSuccess) e = cudaMalloc(&s->block, particles_block_bytes(capacity));
    if (e != cudaSuccess) {
        for (int k = 0; k < 2; ++k) { cudaFree(s->keys[k]); cudaFree(s->vals[k]); }
        cudaFree(s->temp); cudaFree(s->block);
        delete s;
        return cuda_status(e);
    }
    *out = s;
    return FPG_OK;
}

extern "C" fpg_status fpg_sorter_destroy(fpg_sorter* s) {
    if (!s) return FPG_OK;
    for (int k = 0; k < 2; ++k) { cudaFree(s->keys[k]); cudaFree(s->vals[k]); }
    cudaFree(s->temp);
    cudaFree(s->block);
    delete s;
    return FPG_OK;
}

extern "C" fpg_status fpg_sort_by_cell(fpg_ctx* ctx, fpg_particles* P, const fpg_met* met, fpg_sorter* s,
                                       uint32_t* perm_dev, void* stream) {
    if (!ctx || !P || !met || !s) return FPG_ERR_INVALID_ARGUMENT;
    if (s->capacity != P->capacity) return FPG_ERR_LENGTH_MISMATCH;
    if (met->nx * met->ny * met->nz >= (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    const uint32_t n = (uint32_t)P->dispatch;
    if (n == 0) return FPG_OK;
    cudaStream_t st = ctx->pick(stream);
    KeyArgs a;
    a.cell_x = (const int32_t*)P->field[FPG_FIELD_CELL_X];
    a.cell_y = (const int32_t*)P->field[FPG_FIELD_CELL_Y];
    a.pos_x = (const float*)P->field[FPG_FIELD_POS_X];
    a.pos_y = (const float*)P->field[FPG_FIELD_POS_Y];
    a.pos_z = (const float*)P->field[FPG_FIELD_POS_Z];
    a.flags = (const uint32_t*)P->field[FPG_FIELD_FLAGS];
    a.heights = met->heights_dev;
    a.n = n;
    a.nx = (uint32_t)met->nx; a.ny = (uint32_t)met->ny; a.nz = (uint32_t)met->nz;
    a.has_heights = met->heights_set && met->heights[met->nz - 1] > 0.0f;
    a.monotonic = met->monotonic;
    cell_key_kernel<<<(n + 255) / 256, 256, met->nz * sizeof(float), st>>>(a, s->keys[0], s->vals[0]);
    ctx->count();
    FPG_CHECK_LAUNCH();
    cub::DoubleBuffer<uint32_t> kb(s->keys[0], s->keys[1]), vb(s->vals[0], s->vals[1]);
    size_t tb = s->temp_bytes;
    const int bits = key_bits(met->nx * met->ny * met->nz);
    FPG_CUDA(cub::DeviceRadixSort::SortPairs(s->temp, tb, kb, vb, (int)n, 0, bits, st));
    ctx->count(1 + (bits + 7) / 8);  // histogram + one pass per 8-bit digit
    const uint32_t* perm = vb.Current();
    SortFields src, dst;
    void* dst_fields[FPG_FIELD_COUNT];
    particles_assign_fields(s->block, s->capacity, dst_fields);
    for (int f = 0; f < FPG_FIELD_COUNT; ++f) {
        src.f[f] = static_cast<uint32_t*>(P->field[f]);
        dst.f[f] = static_cast<uint32_t*>(dst_fields[f]);
    }
    const uint32_t cap = (uint32_t)P->capacity;
    permute_kernel<<<(cap + 255) / 256, 256, 0, st>>>(src, dst, perm, n, cap);
    ctx->count();
    FPG_CHECK_LAUNCH();
    if (perm_dev) FPG_CUDA(cudaMemcpyAsync(perm_dev, perm, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    particles_swap_block(P, &s->block);
    return FPG_OK;
}
