// slots.cuh — the per-slot view of a particle store shared by the kernels
// that read positions and flags only (Hanna records, CBL sampling).
#pragma once

#include <cstdint>

#include "fpg_internal.h"
#include "physics.cuh"

namespace fpg {

// The kernels move records as 16-byte vectors: device pointers from the
// caller must be 16-byte aligned (cudaMalloc gives 256).
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0u; }

struct SlotView {
    const int32_t* cell_x;
    const int32_t* cell_y;
    const float* pos_x;
    const float* pos_y;
    const float* pos_z;
    const uint32_t* flags;
    size_t n;
};

inline SlotView slot_view(const fpg_particles* P) {
    return SlotView{static_cast<const int32_t*>(P->field[FPG_FIELD_CELL_X]),
                    static_cast<const int32_t*>(P->field[FPG_FIELD_CELL_Y]),
                    static_cast<const float*>(P->field[FPG_FIELD_POS_X]),
                    static_cast<const float*>(P->field[FPG_FIELD_POS_Y]),
                    static_cast<const float*>(P->field[FPG_FIELD_POS_Z]),
                    static_cast<const uint32_t*>(P->field[FPG_FIELD_FLAGS]), P->dispatch};
}

// hanna_params.wgsl:244-250: the PBL cell of the particle's position.
__device__ __forceinline__ uint32_t pbl_cell_index(const SlotView& v, size_t p, uint32_t pnx, uint32_t pny) {
    const float x = (float)v.cell_x[p] + v.pos_x[p];
    const float y = (float)v.cell_y[p] + v.pos_y[p];
    const uint32_t i = (uint32_t)floorf(clampf(x, 0.0f, (float)(pnx - 1u)));
    const uint32_t j = (uint32_t)floorf(clampf(y, 0.0f, (float)(pny - 1u)));
    return i * pny + j;
}

__device__ __forceinline__ float4 pbl_cell(const SlotView& v, size_t p, const float4* pbl, uint32_t pnx,
                                           uint32_t pny) {
    return __ldg(pbl + pbl_cell_index(v, p, pnx, pny));
}

}  // namespace fpg
