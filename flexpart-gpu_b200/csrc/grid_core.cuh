// grid_core.cuh -- level binning and mass quantisation of the concentration
// grid (concentration_gridding.wgsl:304-326), shared by grid.cu and batch.cu.
#pragma once

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

// quantize_mass_to_u32 (concentration_gridding.wgsl:317-326).
__device__ __forceinline__ uint32_t quantize(float m, float scale) {
    if (m <= 0.0f) return 0u;
    const float scaled = m * scale + 0.5f;
    if (scaled >= 4294967295.0f) return 0xffffffffu;
    return (uint32_t)scaled;
}

}  // namespace fpg
