// compact.cu — stable active-particle compaction (compaction.wgsl:65-217,
// host src/gpu/compaction.rs:447-505).
//
// Three kernels over tiles of TILE = 2048 slots (256 threads x 8 slots):
//   1. count:   each warp ballots the active bit of 32 slots at a time and
//               sums popcounts; one count per tile;
//   2. scan:    one block turns tile counts into exclusive offsets and the
//               total (the active count);
//   3. scatter: each active slot goes to offset(tile) + its rank among the
//               active slots before it in the tile (ballot + popc), so the
//               original order is kept; every slot >= active count receives
//               its own old contents with the active bit cleared.
// All FPG_FIELD_COUNT arrays move into a second structure-of-arrays block
// that is then swapped with the particle handle's (no copy back).
#include <cuda_runtime.h>

#include <cstring>

#include "fpg_internal.h"

namespace fpg {

void particles_swap_block(fpg_particles* p, void** other_block);
size_t particles_block_bytes(size_t capacity);
void particles_assign_fields(void* block, size_t capacity, void** field);

constexpr int CT_THREADS = 256;
constexpr int CT_ITEMS = 8;
constexpr int CT_TILE = CT_THREADS * CT_ITEMS;

struct Fields { uint32_t* f[FPG_FIELD_COUNT]; };

// Per-tile active count.  Slot order inside a tile: item-major chunks of 256
// (chunk c covers slots tile*TILE + c*256 .. +255), warp w of the chunk
// covers 32 consecutive slots.
__global__ void __launch_bounds__(CT_THREADS) compact_count_kernel(const uint32_t* __restrict__ flags, uint32_t n,
                                                                   uint32_t* __restrict__ tile_counts) {
    __shared__ uint32_t s_warp[CT_THREADS / 32];
    const uint32_t tile = blockIdx.x;
    uint32_t local = 0;
#pragma unroll
    for (int c = 0; c < CT_ITEMS; ++c) {
        const uint32_t slot = tile * CT_TILE + c * CT_THREADS + threadIdx.x;
        const bool act = slot < n && (flags[slot] & 1u);
        local += __popc(__ballot_sync(0xffffffffu, act));
    }
    if ((threadIdx.x & 31u) == 0) s_warp[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < CT_THREADS / 32; ++w) t += s_warp[w];
        tile_counts[tile] = t;
    }
}

// Exclusive scan of tile counts in one block of 1024 threads; writes the
// total to *active.
__global__ void __launch_bounds__(1024) compact_scan_kernel(uint32_t* __restrict__ tile_counts, uint32_t n_tiles,
                                                            uint32_t* __restrict__ active) {
    __shared__ uint32_t s[1024];
    const uint32_t per = (n_tiles + 1023u) / 1024u;
    const uint32_t begin = threadIdx.x * per;
    const uint32_t end = min(begin + per, n_tiles);
    uint32_t sum = 0;
    for (uint32_t i = begin; i < end; ++i) sum += tile_counts[i];
    s[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024u; off <<= 1) {
        const uint32_t v = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = s[threadIdx.x] - sum;
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t v = tile_counts[i];
        tile_counts[i] = run;
        run += v;
    }
    if (threadIdx.x == 1023u) *active = s[1023];
}

__global__ void __launch_bounds__(CT_THREADS) compact_scatter_kernel(Fields src, Fields dst, uint32_t n,
                                                                     const uint32_t* __restrict__ tile_offsets,
                                                                     const uint32_t* __restrict__ active_ptr,
                                                                     uint32_t* __restrict__ indices) {
    __shared__ uint32_t s_warp[CT_ITEMS][CT_THREADS / 32];
    const uint32_t tile = blockIdx.x;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    unsigned ballots[CT_ITEMS];
#pragma unroll
    for (int c = 0; c < CT_ITEMS; ++c) {
        const uint32_t slot = tile * CT_TILE + c * CT_THREADS + threadIdx.x;
        const bool act = slot < n && (src.f[FPG_FIELD_FLAGS][slot] & 1u);
        ballots[c] = __ballot_sync(0xffffffffu, act);
        if (lane == 0) s_warp[c][warp] = __popc(ballots[c]);
    }
    __syncthreads();
    // exclusive prefix over (chunk, warp) in slot order, computed per thread
    const uint32_t active = *active_ptr;
    uint32_t base = tile_offsets[tile];
#pragma unroll
    for (int c = 0; c < CT_ITEMS; ++c) {
        uint32_t before = base;
        for (unsigned w = 0; w < warp; ++w) before += s_warp[c][w];
        uint32_t chunk_total = 0;
        for (unsigned w = 0; w < CT_THREADS / 32; ++w) chunk_total += s_warp[c][w];
        const uint32_t slot = tile * CT_TILE + c * CT_THREADS + threadIdx.x;
        if (slot < n) {
            if (ballots[c] & (1u << lane)) {
                const uint32_t d = before + __popc(ballots[c] & lt_mask);
#pragma unroll
                for (int f = 0; f < FPG_FIELD_COUNT; ++f) dst.f[f][d] = src.f[f][slot];
                if (indices) indices[d] = slot;
            }
            if (slot >= active) {
#pragma unroll
                for (int f = 0; f < FPG_FIELD_COUNT; ++f) {
                    uint32_t v = src.f[f][slot];
                    if (f == FPG_FIELD_FLAGS) v &= ~1u;
                    dst.f[f][slot] = v;
                }
            }
        }
        base += chunk_total;
    }
}

}  // namespace fpg

using namespace fpg;

extern "C" fpg_status fpg_compaction_create(fpg_ctx* ctx, size_t capacity, fpg_compaction** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (capacity > (size_t)UINT32_MAX - CT_TILE) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_compaction* c = new fpg_compaction();
    c->ctx = ctx;
    c->capacity = capacity;
    c->n_tiles = (capacity + CT_TILE - 1) / CT_TILE;
    cudaError_t e = cudaMalloc(&c->block, particles_block_bytes(capacity));
    if (e == cudaSuccess) e = cudaMalloc(&c->tile_counts, (c->n_tiles > 0 ? c->n_tiles : 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&c->active_count_dev, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&c->active_count_host, sizeof(uint32_t));
    if (e != cudaSuccess) {
        cudaFree(c->block); cudaFree(c->tile_counts); cudaFree(c->active_count_dev);
        if (c->active_count_host) cudaFreeHost(c->active_count_host);
        delete c;
        return cuda_status(e);
    }
    *out = c;
    return FPG_OK;
}

extern "C" fpg_status fpg_compaction_destroy(fpg_compaction* c) {
    if (!c) return FPG_OK;
    cudaFree(c->block);
    cudaFree(c->tile_counts);
    cudaFree(c->active_count_dev);
    cudaFreeHost(c->active_count_host);
    delete c;
    return FPG_OK;
}

extern "C" fpg_status fpg_compact(fpg_ctx* ctx, fpg_particles* P, fpg_compaction* c, uint32_t* active_count,
                                  uint32_t* indices_dev, void* stream) {
    if (!ctx || !P || !c) return FPG_ERR_INVALID_ARGUMENT;
    if (c->capacity != P->capacity) return FPG_ERR_LENGTH_MISMATCH;
    const uint32_t n = (uint32_t)P->capacity;      // compaction.rs:454: all capacity slots
    if (n == 0) {
        if (active_count) *active_count = 0;
        return FPG_OK;
    }
    cudaStream_t s = ctx->pick(stream);
    Fields src, dst;
    void* dst_fields[FPG_FIELD_COUNT];
    particles_assign_fields(c->block, c->capacity, dst_fields);
    for (int f = 0; f < FPG_FIELD_COUNT; ++f) {
        src.f[f] = static_cast<uint32_t*>(P->field[f]);
        dst.f[f] = static_cast<uint32_t*>(dst_fields[f]);
    }
    const uint32_t tiles = (uint32_t)c->n_tiles;
    compact_count_kernel<<<tiles, CT_THREADS, 0, s>>>(src.f[FPG_FIELD_FLAGS], n, c->tile_counts);
    compact_scan_kernel<<<1, 1024, 0, s>>>(c->tile_counts, tiles, c->active_count_dev);
    compact_scatter_kernel<<<tiles, CT_THREADS, 0, s>>>(src, dst, n, c->tile_counts, c->active_count_dev,
                                                         indices_dev);
    ctx->count(3);
    FPG_CHECK_LAUNCH();
    FPG_CUDA(cudaMemcpyAsync(c->active_count_host, c->active_count_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    FPG_CUDA(cudaStreamSynchronize(s));
    particles_swap_block(P, &c->block);
    const uint32_t act = *c->active_count_host;
    P->dispatch = act;                                 // timeloop.rs:1260
    if (active_count) *active_count = act;
    return FPG_OK;
}
