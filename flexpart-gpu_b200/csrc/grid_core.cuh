// grid_core.cuh -- level binning and mass quantisation of the concentration
// grid (concentration_gridding.wgsl:304-326) and the cell-sum machinery of
// the grid kernels (warp runs, per-CTA shared-memory table), shared by
// grid.cu and batch.cu.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace fpg {

// pos_z_to_level (concentration_gridding.wgsl:304-315).
__device__ __forceinline__ uint32_t level_of(float z, const float* h, uint32_t nz, int meters) {
    if (meters) {
        for (uint32_t k = 0; k < nz; ++k)
            if (z <= h[k]) return k;
        return nz - 1u;
    }
    // u32(clamp(i32(floor(z)), 0, nz-1)); float->int conversion saturates
    const int iz = (int)floorf(z);
    return (uint32_t)min(max(iz, 0), (int)nz - 1);
}

// pos_z_to_level for output heights in ascending order, at most
// kSortedLevels of them, branch-free: the first k with z <= h[k] is the
// number of the first nz - 1 heights below z, which `lower` holds padded
// with +inf up to kSortedLevels - 1 entries; a NaN height (no k) is the top
// level, as in the scan.
constexpr uint32_t kSortedLevels = 8;

__device__ __forceinline__ uint32_t level_sorted(float z, const float (&lower)[kSortedLevels - 1], uint32_t nz) {
    uint32_t k = 0;
#pragma unroll
    for (uint32_t i = 0; i < kSortedLevels - 1; ++i) k += lower[i] < z ? 1u : 0u;
    return z == z ? k : nz - 1u;
}

// Host side: whether level_sorted applies to the output heights h[0..nz)
// (metres, ascending, at most kSortedLevels), and its padded table.
inline int sorted_levels(const float* h, uint32_t nz, float (&lower)[kSortedLevels - 1]) {
    int sorted = nz > 0 && nz <= kSortedLevels && h[nz - 1] > 0.0f;
    for (uint32_t k = 1; sorted && k < nz; ++k)
        if (!(h[k] >= h[k - 1])) sorted = 0;
    for (uint32_t k = 0; k < kSortedLevels - 1; ++k) lower[k] = k + 1 < nz ? h[k] : INFINITY;
    return sorted;
}

// quantize_mass_to_u32 (concentration_gridding.wgsl:317-326).
__device__ __forceinline__ uint32_t quantize(float m, float scale) {
    if (m <= 0.0f) return 0u;
    const float scaled = m * scale + 0.5f;
    if (scaled >= 4294967295.0f) return 0xffffffffu;
    return (uint32_t)scaled;
}

// The CTA's table of the cells its chunk touches: open addressing on the
// cell index in shared memory, filled with shared atomics and added to the
// global grid at the end, one pair of atomics per distinct cell per CTA.
constexpr uint32_t kTableBits = 10;
constexpr uint32_t kTable = 1u << kTableBits;             // 1024 entries
constexpr uint32_t kProbes = 8;
constexpr uint32_t kEmpty = 0xffffffffu;   // no cell has this index (cells < 2^32 - 1)

__device__ __forceinline__ void table_add(uint32_t* tk, uint32_t* tc, uint32_t* tm, uint32_t k, uint32_t c,
                                          uint32_t m, uint32_t* __restrict__ counts, uint32_t* __restrict__ mass) {
    uint32_t slot = (k * 2654435761u) >> (32 - kTableBits);
    for (uint32_t i = 0; i < kProbes; ++i) {
        const uint32_t old = atomicCAS(tk + slot, kEmpty, k);
        if (old == kEmpty || old == k) {
            atomicAdd(tc + slot, c);
            atomicAdd(tm + slot, m);
            return;
        }
        slot = (slot + 1u) & (kTable - 1u);
    }
    atomicAdd(counts + k, c);               // crowded table: straight to the grid
    atomicAdd(mass + k, m);
}

// Sums one warp's 32 (cell, scaled mass) pairs by runs of equal cells in
// lane order: a run's last lane holds the run's count (its length) and mass
// (a segmented inclusive scan, five shuffles) and adds them to the table.
// The reorder leaves a warp's cells in a few runs; a cell that appears in
// several runs is simply added several times.  Invalid lanes carry kEmpty
// and add nothing.
__device__ __forceinline__ void warp_runs_add(uint32_t key, uint32_t q, unsigned lane, uint32_t* tk, uint32_t* tc,
                                              uint32_t* tm, uint32_t* __restrict__ counts,
                                              uint32_t* __restrict__ mass) {
    const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
    const uint32_t next = __shfl_down_sync(0xffffffffu, key, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0u || prev != key);
    const unsigned start = 31u - __clz(heads & (0xffffffffu >> (31u - lane)));
    uint32_t v = q;
#pragma unroll
    for (unsigned d = 1; d < 32u; d <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= start + d) v += x;
    }
    if ((lane == 31u || next != key) && key != kEmpty) table_add(tk, tc, tm, key, lane - start + 1u, v, counts, mass);
}

}  // namespace fpg
