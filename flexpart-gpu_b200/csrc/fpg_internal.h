// fpg_internal.h — handle layouts and launch helpers shared by the .cu files
// of libfpg.  Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>

#include "../../include/fpg.h"

namespace fpg {

struct CellHanna;  // physics.cuh: the per-cell Hanna constants (48 bytes)

// Records the CUDA error for fpg_last_cuda_error() and maps it to a status.
fpg_status cuda_status(cudaError_t e);

#define FPG_CUDA(call)                                   \
    do {                                                 \
        cudaError_t fpg_e_ = (call);                     \
        if (fpg_e_ != cudaSuccess) return fpg::cuda_status(fpg_e_); \
    } while (0)

#define FPG_CHECK_LAUNCH() FPG_CUDA(cudaGetLastError())

}  // namespace fpg

struct fpg_ctx {
    int32_t device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    std::atomic<uint64_t> launches{0};
    uint32_t step_shape = 0;                // launch shape of fpg_step (index into its compiled shapes)
    cudaStream_t pick(void* s) const { return s ? static_cast<cudaStream_t>(s) : stream; }
    void count(uint64_t n = 1) { launches.fetch_add(n, std::memory_order_relaxed); }
};

struct fpg_particles {
    fpg_ctx* ctx = nullptr;
    size_t capacity = 0;
    size_t dispatch = 0;
    void* block = nullptr;                  // one allocation, FPG_FIELD_COUNT arrays
    void* field[FPG_FIELD_COUNT] = {};
    // Highest species index + 1 with any non-zero mass ever uploaded.  Slots of
    // higher species are all zero, and zero * survival stays zero, so kernels
    // skip them without changing any result.
    int n_species = 1;
};

// Buckets of the metres->level table (one byte each, staged in shared
// memory beside the level heights by every kernel that searches levels).
constexpr uint32_t FPG_LEVEL_BUCKETS = 1024;

struct fpg_met {
    fpg_ctx* ctx = nullptr;
    size_t nx = 0, ny = 0, nz = 0;
    // Node-major bracket: node n holds (u0, v0, u1, v1, w0, w1, 0, 0) of t0
    // (0) and t1 (1) in bracket[2n], bracket[2n+1]; node n =
    // ((ix*ny)+iy)*nz+iz as in the reference layout.
    float4* bracket = nullptr;
    float* staging = nullptr;               // 3*nodes floats for host uploads
    float* heights_dev = nullptr;           // nz level heights on the device
    float heights[FPG_MAX_LEVELS] = {};
    bool heights_set = false;
    bool monotonic = true;
    // Bucket table of the level search (heights non-decreasing with
    // h[nz-1] > h[0]): bucket b of (z - h[0]) * level_inv_w holds the first
    // level index, minus one, whose height is at least the lower edge of
    // bucket b - 1, so the search scans up from there.
    uint8_t* level_table_dev = nullptr;
    float level_inv_w = 0.0f;
    bool level_table = false;
    bool uploaded[2] = {false, false};
};

// Dynamic shared memory of a kernel that stages the level heights and table.
inline size_t level_smem_bytes(const fpg_met* m) { return m->nz * sizeof(float) + FPG_LEVEL_BUCKETS; }

struct fpg_pbl {
    fpg_ctx* ctx = nullptr;
    size_t nx = 0, ny = 0;
    float* field[7] = {};                   // ustar, wstar, hmix, oli, sshf, ssr, surfstr
    float4* packed = nullptr;               // (ustar, wstar, hmix, oli) per cell
    fpg::CellHanna* hanna = nullptr;        // the Hanna constants of each cell (the fused step reads these)
    bool ready = false;
};

struct fpg_surface {
    fpg_ctx* ctx = nullptr;
    size_t nx = 0, ny = 0;
    fpg_surface_cell* frame[2] = {};
    bool uploaded[2] = {false, false};
};

struct fpg_cellfield {
    fpg_ctx* ctx = nullptr;
    size_t nx = 0, ny = 0;
    float2* lf = nullptr;                   // (lambda, fraction) per cell
    float* staging = nullptr;               // 3*cells floats
    bool ready = false;
};

struct fpg_grid {
    fpg_ctx* ctx = nullptr;
    size_t nx = 0, ny = 0, nz = 0;
    uint32_t* counts = nullptr;
    uint32_t* mass = nullptr;
    float mass_scale = 1.0e6f;
    // fpg_grid_download_async: the copy waits for `produced` (recorded on the
    // stream of the last accumulate); the next accumulate waits for `copied`.
    cudaStream_t last_stream = nullptr;
    cudaEvent_t produced = nullptr;
    cudaEvent_t copied = nullptr;
    bool copy_pending = false;
};

struct fpg_compaction {
    fpg_ctx* ctx = nullptr;
    size_t capacity = 0;
    void* block = nullptr;                  // second structure-of-arrays (swapped in)
    uint32_t* tile_counts = nullptr;        // per-tile active counts, then offsets
    uint32_t* active_count_dev = nullptr;
    uint32_t* active_count_host = nullptr;  // pinned
    size_t n_tiles = 0;
};
