// compact_static.cu — the stable compaction scan with no allocation at all.
//
// Some callers of this library cannot call cudaMalloc: a host program whose
// device memory is owned by someone else (a framework's caching allocator, or
// an arena carved out once at start-up) and that forbids libraries from
// allocating on their own, or a latency-critical loop where an allocation
// would synchronise the device.  fpg_compact needs per-call scratch (the
// per-tile counts) that its handle allocates up front; this entry point keeps
// that scratch in a file-scope static device array instead, so the caller
// passes only its own input and output buffers.
//
// It computes what the first three passes of the reference compaction compute
// (compaction.wgsl:65-185): the original slot of each active particle, in slot
// order, and the active count.  It does not move particle data.
//
// Limits and sharing:
//   * at most FPG_STATIC_COMPACT_MAX_SLOTS slots per call (65536 tiles of
//     2048 slots); larger calls return FPG_ERR_VALUE_TOO_LARGE;
//   * the array (256 KiB) lives on every GPU that loads this library until
//     the process exits;
//   * every call shares the one array per device: calls whose work overlaps
//     on the GPU (different streams, no ordering between them) race and
//     corrupt each other's counts.  Calls ordered on one stream are safe;
//   * each call writes every scratch entry it reads before reading it, so
//     stale contents from an earlier call never leak into a result.
//
// In host code the array's name is only a host-side stand-in; its device
// address is looked up with cudaGetSymbolAddress once per device (with that
// device current) on the first call made for a context on that device, and
// cached.  That first call should therefore come before any stream capture.
// The cached address belongs to the device's primary context as it was at
// that first call: a cudaDeviceReset on that device ends the context and the
// module with it, and this entry point must not be called again in that
// process after such a reset.
#include <cuda_runtime.h>

#include <mutex>

#include "fpg_internal.h"

namespace fpg {
namespace {

constexpr int ST_THREADS = 256;
constexpr int ST_ITEMS = 8;
constexpr int ST_TILE = ST_THREADS * ST_ITEMS;
constexpr uint32_t ST_MAX_TILES = FPG_STATIC_COMPACT_MAX_SLOTS / ST_TILE;
constexpr int ST_MAX_DEVICES = 64;

static __device__ __align__(256) uint32_t g_tile_scratch[ST_MAX_TILES];

std::mutex g_setup_mutex;
uint32_t* g_scratch_dev[ST_MAX_DEVICES] = {};

// Device address of g_tile_scratch on `device`, looked up once per device.
fpg_status scratch_for(int device, uint32_t** out) {
    if (device < 0 || device >= ST_MAX_DEVICES) return FPG_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[device]) {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return cuda_status(e);
        if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return cuda_status(e);
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_tile_scratch);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess) return cuda_status(e);
        g_scratch_dev[device] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_dev[device];
    return FPG_OK;
}

__global__ void __launch_bounds__(ST_THREADS) static_count_kernel(const uint32_t* __restrict__ flags, uint32_t n,
                                                                  uint32_t* __restrict__ tiles) {
    __shared__ uint32_t s_warp[ST_THREADS / 32];
    uint32_t local = 0;
#pragma unroll
    for (int c = 0; c < ST_ITEMS; ++c) {
        const uint32_t slot = blockIdx.x * ST_TILE + c * ST_THREADS + threadIdx.x;
        local += __popc(__ballot_sync(0xffffffffu, slot < n && (flags[slot] & 1u)));
    }
    if ((threadIdx.x & 31u) == 0) s_warp[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < ST_THREADS / 32; ++w) t += s_warp[w];
        tiles[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) static_scan_kernel(uint32_t* __restrict__ tiles, uint32_t n_tiles,
                                                           uint32_t* __restrict__ active) {
    __shared__ uint32_t s[1024];
    const uint32_t per = (n_tiles + 1023u) / 1024u;
    const uint32_t begin = threadIdx.x * per;
    const uint32_t end = min(begin + per, n_tiles);
    uint32_t sum = 0;
    for (uint32_t i = begin; i < end; ++i) sum += tiles[i];
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
        const uint32_t v = tiles[i];
        tiles[i] = run;
        run += v;
    }
    if (threadIdx.x == 1023u) *active = s[1023];
}

__global__ void __launch_bounds__(ST_THREADS) static_index_kernel(const uint32_t* __restrict__ flags, uint32_t n,
                                                                  const uint32_t* __restrict__ offsets,
                                                                  uint32_t* __restrict__ indices) {
    __shared__ uint32_t s_warp[ST_ITEMS][ST_THREADS / 32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned ballots[ST_ITEMS];
#pragma unroll
    for (int c = 0; c < ST_ITEMS; ++c) {
        const uint32_t slot = blockIdx.x * ST_TILE + c * ST_THREADS + threadIdx.x;
        ballots[c] = __ballot_sync(0xffffffffu, slot < n && (flags[slot] & 1u));
        if (lane == 0) s_warp[c][warp] = __popc(ballots[c]);
    }
    __syncthreads();
    uint32_t base = offsets[blockIdx.x];
#pragma unroll
    for (int c = 0; c < ST_ITEMS; ++c) {
        uint32_t before = base, chunk = 0;
        for (unsigned w = 0; w < ST_THREADS / 32; ++w) {
            if (w < warp) before += s_warp[c][w];
            chunk += s_warp[c][w];
        }
        if (ballots[c] & (1u << lane))
            indices[before + __popc(ballots[c] & ((1u << lane) - 1u))] = blockIdx.x * ST_TILE + c * ST_THREADS + threadIdx.x;
        base += chunk;
    }
}

}  // namespace
}  // namespace fpg

using namespace fpg;

extern "C" fpg_status fpg_compaction_indices_static(fpg_ctx* ctx, const uint32_t* flags_dev, size_t n,
                                                    uint32_t* indices_dev, uint32_t* active_count_dev,
                                                    void* stream) {
    if (!ctx || !active_count_dev || (n && (!flags_dev || !indices_dev))) return FPG_ERR_INVALID_ARGUMENT;
    if (n > (size_t)FPG_STATIC_COMPACT_MAX_SLOTS) return FPG_ERR_VALUE_TOO_LARGE;
    uint32_t* tiles = nullptr;
    fpg_status st = scratch_for(ctx->device, &tiles);
    if (st != FPG_OK) return st;
    cudaStream_t s = ctx->pick(stream);
    if (n == 0) {
        FPG_CUDA(cudaMemsetAsync(active_count_dev, 0, sizeof(uint32_t), s));
        return FPG_OK;
    }
    const uint32_t n_tiles = (uint32_t)((n + ST_TILE - 1) / ST_TILE);
    static_count_kernel<<<n_tiles, ST_THREADS, 0, s>>>(flags_dev, (uint32_t)n, tiles);
    static_scan_kernel<<<1, 1024, 0, s>>>(tiles, n_tiles, active_count_dev);
    static_index_kernel<<<n_tiles, ST_THREADS, 0, s>>>(flags_dev, (uint32_t)n, tiles, indices_dev);
    ctx->count(3);
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}
