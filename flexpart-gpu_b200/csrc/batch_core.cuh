// batch_core.cuh — the batched ensemble's device state and host handle,
// shared by the batched step (batch.cu) and the source inversion built on it
// (adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/fpg_driver.h"
#include "fpg_internal.h"
#include "physics.cuh"
#include "step_core.cuh"

namespace fpg {

constexpr uint32_t TILE = 256;
constexpr uint32_t kNumVariants = 11;  // compiled launch shapes of the particle pass

struct BatchState {
    int64_t t;
    int64_t ta;
    uint32_t step;
    int32_t fa, fb;
    int32_t have_bracket;
    int32_t changed;
    float alpha;
    int32_t error;
    uint32_t work;
};

struct ScenDev {
    uint32_t offset, capacity, first_tile, n_tiles;
    uint32_t instance;               // source-inversion instance (0 outside inversions)
    uint32_t key0, key1;
    u32x4 counter;
    uint32_t released, rel_lo, rel_hi;
    float mass_per_particle;
    int64_t start, end;
    double lon_min, lon_max, lat_min, lat_max, z_min, z_max;
    uint64_t count;
    uint64_t lat_nx, lat_nxy, lat_nz;
};

struct BatchConst {
    int64_t start, frame_seconds, dt;
    uint32_t n_frames;
    uint32_t n_scen;
    uint32_t n_tiles;
    uint32_t bpp;
    double xlon0, ylat0, dx, dy;
    uint64_t gnx, gny;
};

struct PopFields { uint32_t* f[FPG_FIELD_COUNT]; };

// ReleaseState::target_emitted_count (release/mod.rs:181-196); counts and
// window lengths are below 2^32 (checked at create), so the u128 product of
// the reference fits in 64 bits.
__host__ __device__ inline uint32_t target_emitted(int64_t start, int64_t end, uint64_t count, int64_t now,
                                                   uint32_t released) {
    if (now < start || now > end) return released;
    if (start == end) return (uint32_t)count;
    if (now == end) return (uint32_t)count;
    return (uint32_t)((count * (uint64_t)(now - start)) / (uint64_t)(end - start));
}

__host__ __device__ inline u32x4 counter_add64(u32x4 c, uint64_t off) {
    // philox_counter_add (rng.rs:69-87)
    const uint32_t lo = (uint32_t)off, hi = (uint32_t)(off >> 32);
    u32x4 r;
    r.x = c.x + lo;
    const uint32_t carry0 = r.x < c.x;
    const uint32_t n1 = c.y + hi;
    const uint32_t carry1a = n1 < c.y;
    r.y = n1 + carry0;
    const uint32_t carry1b = r.y < n1;
    r.z = c.z + (carry1a | carry1b);
    const uint32_t carry2 = r.z < c.z;
    r.w = c.w + carry2;
    return r;
}

struct InverseData;

}  // namespace fpg

struct fpg_batch {
    fpg_ctx* ctx = nullptr;
    fpg_batch_config cfg{};
    std::vector<float> outheights;
    std::vector<fpg::ScenDev> scen;            // host copy at creation / host mirror for the sequential path
    std::vector<uint32_t> tile_scen_h;
    size_t capacity = 0;
    uint32_t n_tiles = 0;
    uint64_t total_steps = 0, steps_done = 0;
    fpg_particles* pop = nullptr;
    fpg_met* met = nullptr;
    fpg_pbl* pbl = nullptr;
    fpg_cellfield* wet = nullptr;
    float4* ring = nullptr;               // n_frames * nodes packed (u,v,w,0)
    fpg_surface_cell* sring = nullptr;    // n_frames * cells
    float* pring = nullptr;               // n_frames * cells precipitation
    float* staging = nullptr;             // 3 * nodes
    fpg::BatchState* st = nullptr;
    fpg::ScenDev* sc = nullptr;
    uint32_t* tile_scen = nullptr;
    uint2* items = nullptr;               // work items of the chosen launch shape
    uint32_t n_items = 0;
    size_t items_cap = 0;
    uint32_t variant = 0;                 // index into kVariants
    uint32_t resident[fpg::kNumVariants] = {}; // CTAs per SM of each shape (occupancy API)
    float tuned_ms = 0.0f;
    uint32_t* grid_counts = nullptr;
    uint32_t* grid_mass = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t graph_launches = 0;          // kernels in one replay of the step graph
    std::vector<uint32_t> released_h;     // host mirror of the release counts (sequential path)
    std::vector<fpg::u32x4> counter_h;
    int64_t t_h = 0;
    fpg::InverseData* inv = nullptr;      // set by a source inversion built on this batch
};


namespace fpg {

StepArgs make_step_args(fpg_batch* b);
BatchConst make_const(const fpg_batch* b);
PopFields pop_fields(fpg_batch* b);
// Per-step kernels before the particle pass (clock, bracket, PBL, release),
// the particle pass in the chosen launch shape, and the kernels after it
// (grids, inversion sampling, counter and clock advance).
void enqueue_pre(fpg_batch* b, cudaStream_t s);
void enqueue_step_kernel(fpg_batch* b, cudaStream_t s);
void enqueue_post(fpg_batch* b, cudaStream_t s);
// Repacks the bracket of state st's frames whether or not it changed.
void enqueue_pack_forced(fpg_batch* b, const BatchState* st, cudaStream_t s);
fpg_status build_items(fpg_batch* b, uint32_t variant);
// The counter and clock advance alone (batch_end_kernel).
void enqueue_end(fpg_batch* b, cudaStream_t s);
// Captures the step graph (pre, particle pass, post) if none is held.
fpg_status ensure_graph(fpg_batch* b);
// FPG_ERR_OUT_OF_GRID when the scenario's release lattice leaves the grid.
fpg_status check_release_grid(const ScenDev& d, const fpg_grid_domain& g);
size_t particles_block_bytes(size_t capacity);
// Back to the start time: population zeroed, nothing released, the
// scenarios' initial counters, no bracket on the device.
fpg_status batch_reset(fpg_batch* b);
// Receptor sampling of a source inversion at output steps (adjoint.cu).
void enqueue_inverse_sample(fpg_batch* b, cudaStream_t s);

}  // namespace fpg
