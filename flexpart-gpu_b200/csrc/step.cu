// step.cu — the fused per-particle step and the per-cell kernels around it.
//
// fused_step_kernel is the B200 replacement of four reference compute passes
// encoded back to back by ForwardTimeLoopDriver::run_timestep
// (src/simulation/timeloop.rs:1095-1180):
//   advection_dual_wind.wgsl:254-303  (Petterssen with dual-time wind)
//   langevin_fused.wgsl:402-518        (Hanna + Langevin, sub-steps, reflection)
//   dry_deposition.wgsl:76-106         (mass decay in the surface layer)
//   wet_deposition.wgsl:190-217        (below-cloud scavenging)
// Each reference pass reads and writes the whole 96-byte particle; here each
// particle's structure-of-arrays fields are read once and written once
// (96 B per particle-step with one species), and the four passes' math runs
// in registers in between.
//
// Data layout in HBM:
//   particles: one 4-byte array per field, slot-indexed (coalesced 128-B
//     warp accesses);
//   wind bracket: node-major, 32 bytes per node (u0, v0, u1, v1, w0, w1,
//     0, 0) of both frames, so the 8 corners of a sample cost 8 32-byte
//     loads and the channels pair up for the packed FP32 lerps;
//   PBL: float4 (u*, w*, hmix, 1/L) per met cell, one 16-byte gather per
//     particle;
//   wet forcing per cell: float2 (lambda, fraction).
// Level heights sit in shared memory beside a 1024-bucket table of level
// indices; for non-decreasing heights the metres->level search reads the
// bucket's entry and scans up from it (same first index as the reference's
// linear scan, advection_dual_wind.wgsl:94-117), else it runs the scan.
//
// The separated Hanna-record -> Langevin path (fpg_dispatch_hanna_params,
// fpg_langevin_with_hanna) lives here too: it must give the fused kernel's
// bits, so it is built with the same division (this unit's compile flags).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "fpg_internal.h"
#include "physics.cuh"
#include "slots.cuh"
#include "step_core.cuh"

namespace fpg {

__global__ void __launch_bounds__(256, 5) fused_step_kernel(StepArgs a) {
    const Levels lv = global_levels(a);
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    particle_step(a, lv, p, p, a.alpha, a.counter, a.key0, a.key1);
}

// The same pass under another launch shape: BLOCK threads per CTA compiled
// for MINB resident CTAs per SM, PPT particles per thread (slots of one CTA
// are contiguous; thread t takes t, t + BLOCK, ...); with several particles
// per thread the CTA stages the level heights in shared memory once (the
// global pointers would cost registers across the loop).  Each particle's
// arithmetic is the same, so the results are too.
template <int BLOCK, int MINB, int PPT>
__global__ void __launch_bounds__(BLOCK, MINB) fused_step_shape_kernel(StepArgs a) {
    extern __shared__ float s_levels[];
    Levels lv{};
    if constexpr (PPT == 1) {
        lv = global_levels(a);
    } else if (a.stages & FPG_STAGE_ADVECT) {
        lv = stage_levels(a, s_levels);
        __syncthreads();
    }
    const size_t base = (size_t)blockIdx.x * (BLOCK * PPT) + threadIdx.x;
#pragma unroll 1
    for (int j = 0; j < PPT; ++j) {
        const size_t p = base + (size_t)j * BLOCK;
        if (p < a.n) particle_step(a, lv, (uint32_t)p, (uint32_t)p, a.alpha, a.counter, a.key0, a.key1);
    }
}

struct StepShape {
    uint32_t block, minb, ppt;
    void (*kernel)(StepArgs);
};

// Shape 0 is fused_step_kernel itself (the default).
const StepShape kStepShapes[] = {
    {256, 5, 1, fused_step_kernel},
    {256, 4, 1, fused_step_shape_kernel<256, 4, 1>},
    {128, 10, 1, fused_step_shape_kernel<128, 10, 1>},
    {256, 5, 2, fused_step_shape_kernel<256, 5, 2>},
    {256, 5, 4, fused_step_shape_kernel<256, 5, 4>},
    {512, 2, 1, fused_step_shape_kernel<512, 2, 1>},
    {256, 6, 1, fused_step_shape_kernel<256, 6, 1>},
    {128, 12, 1, fused_step_shape_kernel<128, 12, 1>},
    {256, 6, 2, fused_step_shape_kernel<256, 6, 2>},
};
constexpr uint32_t kNumStepShapes = sizeof(kStepShapes) / sizeof(kStepShapes[0]);

// ---- per-cell kernels --------------------------------------------------------

__global__ void __launch_bounds__(256) pbl_diag_kernel(const fpg_surface_cell* __restrict__ s0,
                                                       const fpg_surface_cell* __restrict__ s1, float alpha,
                                                       fpg_pbl_options o, uint32_t ncell, float* ustar_o,
                                                       float* wstar_o, float* hmix_o, float* oli_o, float* sshf_o,
                                                       float* ssr_o, float* surfstr_o, float4* packed,
                                                       CellHanna* hanna) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    pbl_cell(s0, s1, alpha, o, c, ustar_o, wstar_o, hmix_o, oli_o, sshf_o, ssr_o, surfstr_o, packed, hanna);
}

__global__ void __launch_bounds__(256) pack_pbl_kernel(const float* __restrict__ u, const float* __restrict__ w,
                                                       const float* __restrict__ h, const float* __restrict__ o,
                                                       uint32_t ncell, float4* packed, CellHanna* hanna) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    packed[c] = make_float4(u[c], w[c], h[c], o[c]);
    st_cell_hanna(hanna + c, cell_hanna(u[c], w[c], obukhov_from_inverse(o[c]), h[c]));
}

__global__ void __launch_bounds__(256) pack_frame_kernel(const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, uint32_t nodes, int which,
                                                         float4* bracket) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    // one frame's lanes of the node (u0, v0, u1, v1, w0, w1, 0, 0)
    if (n >= nodes) return;
    float* node = reinterpret_cast<float*>(bracket + 2u * n);
    reinterpret_cast<float2*>(node)[which] = make_float2(u[n], v[n]);
    node[4 + which] = w[n];
}

// Both frames of a bracket into whole nodes: 24 B read and 32 B written per
// node, where two pack_frame_kernel passes each read the node's other lanes
// back before their partial stores.
__global__ void __launch_bounds__(256) pack_bracket_kernel(const float* __restrict__ u0, const float* __restrict__ v0,
                                                           const float* __restrict__ w0, const float* __restrict__ u1,
                                                           const float* __restrict__ v1, const float* __restrict__ w1,
                                                           uint32_t nodes, float4* bracket) {
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes) return;
    st_node(bracket, n, make_float4(u0[n], v0[n], w0[n], 0.0f), make_float4(u1[n], v1[n], w1[n], 0.0f));
}

// wet_precipitation_state + below_cloud_scavenging_coefficient_gas
// (physics/wet_scavenging.rs:179-225,78-82) per met cell.
__global__ void __launch_bounds__(256) wet_cells_kernel(const float* __restrict__ lsp_in,
                                                        const float* __restrict__ conv_in,
                                                        const float* __restrict__ cc_in, float a_in, float b_in,
                                                        uint32_t ncell, float2* out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    out[c] = wet_cell_forcing(lsp_in[c], conv_in[c], cc_in[c], a_in, b_in);
}

__global__ void __launch_bounds__(256) fill_kernel(float* out, uint32_t n, float v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v;
}

__global__ void __launch_bounds__(256) philox_kernel(uint32_t k0, uint32_t k1, u32x4 base, uint32_t n_blocks,
                                                     float* out, uint32_t* raw) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_blocks) return;
    // philox_rng.wgsl: block b uses counter base + b (64-bit add as rng.rs:69-87)
    u32x4 c = counter_add(base, b);
    const u32x4 r = philox4x32_10(c, k0, k1);
    if (out) {
        out[4u * b + 0u] = u32_to_uniform01(r.x); out[4u * b + 1u] = u32_to_uniform01(r.y);
        out[4u * b + 2u] = u32_to_uniform01(r.z); out[4u * b + 3u] = u32_to_uniform01(r.w);
    }
    if (raw) { raw[4u * b] = r.x; raw[4u * b + 1u] = r.y; raw[4u * b + 2u] = r.z; raw[4u * b + 3u] = r.w; }
}

static inline uint32_t blocks_for(size_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

}  // namespace fpg

using namespace fpg;

// ============================================================================
// C ABI: met, PBL, surface, cell fields
// ============================================================================

extern "C" fpg_status fpg_met_create(fpg_ctx* ctx, size_t nx, size_t ny, size_t nz, fpg_met** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (nx == 0 || ny == 0 || nz == 0) return FPG_ERR_ZERO_SHAPE;
    if (nz > FPG_MAX_LEVELS) return FPG_ERR_TOO_MANY_LEVELS;
    const size_t nodes = nx * ny * nz;
    if (nodes * 2 >= (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_met* m = new fpg_met();
    m->ctx = ctx; m->nx = nx; m->ny = ny; m->nz = nz;
    cudaError_t e = cudaMalloc(&m->bracket, nodes * 2 * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&m->staging, nodes * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->heights_dev, nz * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->level_table_dev, FPG_LEVEL_BUCKETS);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->bracket, 0, nodes * 2 * sizeof(float4), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->heights_dev, 0, nz * sizeof(float), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(m->bracket); cudaFree(m->staging); cudaFree(m->heights_dev); cudaFree(m->level_table_dev);
        delete m;
        return cuda_status(e);
    }
    *out = m;
    return FPG_OK;
}

extern "C" fpg_status fpg_met_destroy(fpg_met* m) {
    if (!m) return FPG_OK;
    cudaFree(m->bracket);
    cudaFree(m->staging);
    cudaFree(m->heights_dev);
    cudaFree(m->level_table_dev);
    delete m;
    return FPG_OK;
}

static fpg_status met_pack(fpg_met* m, int which, const float* u, const float* v, const float* w, cudaStream_t s) {
    const uint32_t nodes = (uint32_t)(m->nx * m->ny * m->nz);
    pack_frame_kernel<<<blocks_for(nodes, 256), 256, 0, s>>>(u, v, w, nodes, which, m->bracket);
    m->ctx->count();
    FPG_CHECK_LAUNCH();
    m->uploaded[which] = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_met_upload_frame(fpg_met* m, int32_t which, const float* u, const float* v,
                                           const float* w, void* stream) {
    if (!m || !u || !v || !w || (which != 0 && which != 1)) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = m->ctx->pick(stream);
    const size_t nodes = m->nx * m->ny * m->nz;
    FPG_CUDA(cudaMemcpyAsync(m->staging, u, nodes * sizeof(float), cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(m->staging + nodes, v, nodes * sizeof(float), cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(m->staging + 2 * nodes, w, nodes * sizeof(float), cudaMemcpyHostToDevice, s));
    return met_pack(m, which, m->staging, m->staging + nodes, m->staging + 2 * nodes, s);
}

extern "C" fpg_status fpg_met_upload_frame_device(fpg_met* m, int32_t which, const float* u, const float* v,
                                                  const float* w, void* stream) {
    if (!m || !u || !v || !w || (which != 0 && which != 1)) return FPG_ERR_INVALID_ARGUMENT;
    return met_pack(m, which, u, v, w, m->ctx->pick(stream));
}

extern "C" fpg_status fpg_met_upload_bracket_device(fpg_met* m, const float* u0, const float* v0, const float* w0,
                                                    const float* u1, const float* v1, const float* w1,
                                                    void* stream) {
    if (!m || !u0 || !v0 || !w0 || !u1 || !v1 || !w1) return FPG_ERR_INVALID_ARGUMENT;
    const uint32_t nodes = (uint32_t)(m->nx * m->ny * m->nz);
    pack_bracket_kernel<<<blocks_for(nodes, 256), 256, 0, m->ctx->pick(stream)>>>(u0, v0, w0, u1, v1, w1, nodes,
                                                                                   m->bracket);
    m->ctx->count();
    FPG_CHECK_LAUNCH();
    m->uploaded[0] = m->uploaded[1] = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_met_set_level_heights(fpg_met* m, const float* heights, size_t n) {
    if (!m || (!heights && n)) return FPG_ERR_INVALID_ARGUMENT;
    if (n > FPG_MAX_LEVELS) return FPG_ERR_TOO_MANY_LEVELS;
    if (n != m->nz) return FPG_ERR_LENGTH_MISMATCH;
    std::memcpy(m->heights, heights, n * sizeof(float));
    m->monotonic = true;
    for (size_t k = 1; k < n; ++k)
        if (!(heights[k] >= heights[k - 1])) m->monotonic = false;
    // the bucket table of the level search: entry b is the first level (minus
    // one) at or above the lower edge of bucket b - 1, in double, so that any
    // z whose float bucket index is b lies above every level below it
    uint8_t table[FPG_LEVEL_BUCKETS];
    m->level_table = m->monotonic && n >= 2 && heights[n - 1] > heights[0] && std::isfinite(heights[0]) &&
                     std::isfinite(heights[n - 1]);
    if (m->level_table) {
        const double h0 = heights[0], span = (double)heights[n - 1] - h0, w = span / FPG_LEVEL_BUCKETS;
        m->level_inv_w = (float)(FPG_LEVEL_BUCKETS / span);
        size_t k = 1;
        for (uint32_t b = 0; b < FPG_LEVEL_BUCKETS; ++b) {
            const double edge = h0 + ((double)b - 1.0) * w;
            while (k < n && (double)heights[k] < edge) ++k;
            table[b] = (uint8_t)(k - 1);
        }
        FPG_CUDA(cudaMemcpyAsync(m->level_table_dev, table, FPG_LEVEL_BUCKETS, cudaMemcpyHostToDevice,
                                 m->ctx->stream));
    }
    FPG_CUDA(cudaMemcpyAsync(m->heights_dev, m->heights, n * sizeof(float), cudaMemcpyHostToDevice, m->ctx->stream));
    FPG_CUDA(cudaStreamSynchronize(m->ctx->stream));
    m->heights_set = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_pbl_create(fpg_ctx* ctx, size_t nx, size_t ny, fpg_pbl** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (nx == 0 || ny == 0) return FPG_ERR_ZERO_SHAPE;
    if (nx * ny >= (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_pbl* p = new fpg_pbl();
    p->ctx = ctx; p->nx = nx; p->ny = ny;
    const size_t n = nx * ny;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 7 && e == cudaSuccess; ++k) e = cudaMalloc(&p->field[k], n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&p->packed, n * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&p->hanna, n * sizeof(CellHanna));
    if (e != cudaSuccess) {
        for (int k = 0; k < 7; ++k) cudaFree(p->field[k]);
        cudaFree(p->packed);
        cudaFree(p->hanna);
        delete p;
        return cuda_status(e);
    }
    *out = p;
    return FPG_OK;
}

extern "C" fpg_status fpg_pbl_destroy(fpg_pbl* p) {
    if (!p) return FPG_OK;
    for (int k = 0; k < 7; ++k) cudaFree(p->field[k]);
    cudaFree(p->packed);
    cudaFree(p->hanna);
    delete p;
    return FPG_OK;
}

extern "C" fpg_status fpg_pbl_upload(fpg_pbl* p, const float* ustar, const float* wstar, const float* hmix,
                                     const float* oli, const float* sshf, const float* ssr, const float* surfstr,
                                     void* stream) {
    if (!p || !ustar || !wstar || !hmix || !oli) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = p->ctx->pick(stream);
    const size_t n = p->nx * p->ny;
    const float* src[7] = {ustar, wstar, hmix, oli, sshf, ssr, surfstr};
    for (int k = 0; k < 7; ++k) {
        if (src[k]) FPG_CUDA(cudaMemcpyAsync(p->field[k], src[k], n * sizeof(float), cudaMemcpyHostToDevice, s));
        else FPG_CUDA(cudaMemsetAsync(p->field[k], 0, n * sizeof(float), s));
    }
    pack_pbl_kernel<<<blocks_for(n, 256), 256, 0, s>>>(p->field[0], p->field[1], p->field[2], p->field[3],
                                                        (uint32_t)n, p->packed, p->hanna);
    p->ctx->count();
    FPG_CHECK_LAUNCH();
    p->ready = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_pbl_download(fpg_pbl* p, float* ustar, float* wstar, float* hmix, float* oli, float* sshf,
                                       float* ssr, float* surfstr, void* stream) {
    if (!p) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = p->ctx->pick(stream);
    const size_t n = p->nx * p->ny;
    float* dst[7] = {ustar, wstar, hmix, oli, sshf, ssr, surfstr};
    for (int k = 0; k < 7; ++k)
        if (dst[k]) FPG_CUDA(cudaMemcpyAsync(dst[k], p->field[k], n * sizeof(float), cudaMemcpyDeviceToHost, s));
    FPG_CUDA(cudaStreamSynchronize(s));
    return FPG_OK;
}

extern "C" fpg_status fpg_surface_create(fpg_ctx* ctx, size_t nx, size_t ny, fpg_surface** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (nx == 0 || ny == 0) return FPG_ERR_ZERO_SHAPE;
    if (nx * ny >= (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_surface* s = new fpg_surface();
    s->ctx = ctx; s->nx = nx; s->ny = ny;
    cudaError_t e = cudaMalloc(&s->frame[0], nx * ny * sizeof(fpg_surface_cell));
    if (e == cudaSuccess) e = cudaMalloc(&s->frame[1], nx * ny * sizeof(fpg_surface_cell));
    if (e != cudaSuccess) {
        cudaFree(s->frame[0]); cudaFree(s->frame[1]); delete s;
        return cuda_status(e);
    }
    *out = s;
    return FPG_OK;
}

extern "C" fpg_status fpg_surface_destroy(fpg_surface* s) {
    if (!s) return FPG_OK;
    cudaFree(s->frame[0]);
    cudaFree(s->frame[1]);
    delete s;
    return FPG_OK;
}

extern "C" fpg_status fpg_surface_upload(fpg_surface* s, int32_t which, const fpg_surface_cell* cells, void* stream) {
    if (!s || !cells || (which != 0 && which != 1)) return FPG_ERR_INVALID_ARGUMENT;
    // host or device memory (the copy kind follows the pointer, unified addressing)
    FPG_CUDA(cudaMemcpyAsync(s->frame[which], cells, s->nx * s->ny * sizeof(fpg_surface_cell),
                             cudaMemcpyDefault, s->ctx->pick(stream)));
    s->uploaded[which] = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_pbl_diagnostics(fpg_ctx* ctx, const fpg_surface* surface, float alpha,
                                          const fpg_pbl_options* options, fpg_pbl* pbl, void* stream) {
    if (!ctx || !surface || !options || !pbl) return FPG_ERR_INVALID_ARGUMENT;
    if (surface->nx != pbl->nx || surface->ny != pbl->ny) return FPG_ERR_SHAPE_MISMATCH;
    if (!surface->uploaded[0] || !surface->uploaded[1]) return FPG_ERR_NOT_READY;
    cudaStream_t s = ctx->pick(stream);
    const uint32_t n = (uint32_t)(pbl->nx * pbl->ny);
    // 64-thread CTAs spread the cells over more SMs (one cell per thread, a long dependent chain each)
    pbl_diag_kernel<<<blocks_for(n, 64), 64, 0, s>>>(surface->frame[0], surface->frame[1], alpha, *options, n,
                                                        pbl->field[0], pbl->field[1], pbl->field[2], pbl->field[3],
                                                        pbl->field[4], pbl->field[5], pbl->field[6], pbl->packed,
                                                        pbl->hanna);
    ctx->count();
    FPG_CHECK_LAUNCH();
    pbl->ready = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_cellfield_create(fpg_ctx* ctx, size_t nx, size_t ny, fpg_cellfield** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (nx == 0 || ny == 0) return FPG_ERR_ZERO_SHAPE;
    if (nx * ny >= (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_cellfield* f = new fpg_cellfield();
    f->ctx = ctx; f->nx = nx; f->ny = ny;
    cudaError_t e = cudaMalloc(&f->lf, nx * ny * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&f->staging, nx * ny * 3 * sizeof(float));
    if (e != cudaSuccess) {
        cudaFree(f->lf); cudaFree(f->staging); delete f;
        return cuda_status(e);
    }
    *out = f;
    return FPG_OK;
}

extern "C" fpg_status fpg_cellfield_destroy(fpg_cellfield* f) {
    if (!f) return FPG_OK;
    cudaFree(f->lf);
    cudaFree(f->staging);
    delete f;
    return FPG_OK;
}

extern "C" fpg_status fpg_cellfield_upload(fpg_cellfield* f, const float* lambda, const float* fraction,
                                           void* stream) {
    if (!f || !lambda || !fraction) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = f->ctx->pick(stream);
    const size_t n = f->nx * f->ny;
    // interleave on the device: (lambda, fraction) pairs
    FPG_CUDA(cudaMemcpy2DAsync(f->lf, sizeof(float2), lambda, sizeof(float), sizeof(float), n,
                               cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpy2DAsync(reinterpret_cast<float*>(f->lf) + 1, sizeof(float2), fraction, sizeof(float),
                               sizeof(float), n, cudaMemcpyHostToDevice, s));
    f->ready = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_cellfield_from_precipitation(fpg_cellfield* f, const float* lsp, const float* convp,
                                                       const float* cloud_cover, float a, float b, void* stream) {
    if (!f) return FPG_ERR_INVALID_ARGUMENT;
    cudaStream_t s = f->ctx->pick(stream);
    const size_t n = f->nx * f->ny;
    float* d_lsp = f->staging;
    float* d_conv = f->staging + n;
    float* d_cc = f->staging + 2 * n;
    // host or device arrays (the copy kind follows the pointer, unified addressing)
    if (lsp) FPG_CUDA(cudaMemcpyAsync(d_lsp, lsp, n * sizeof(float), cudaMemcpyDefault, s));
    else FPG_CUDA(cudaMemsetAsync(d_lsp, 0, n * sizeof(float), s));
    if (convp) FPG_CUDA(cudaMemcpyAsync(d_conv, convp, n * sizeof(float), cudaMemcpyDefault, s));
    else FPG_CUDA(cudaMemsetAsync(d_conv, 0, n * sizeof(float), s));
    if (cloud_cover) {
        FPG_CUDA(cudaMemcpyAsync(d_cc, cloud_cover, n * sizeof(float), cudaMemcpyDefault, s));
    } else {
        fill_kernel<<<blocks_for(n, 256), 256, 0, s>>>(d_cc, (uint32_t)n, 1.0f);  // cloud cover 1
        f->ctx->count();
        FPG_CHECK_LAUNCH();
    }
    wet_cells_kernel<<<blocks_for(n, 256), 256, 0, s>>>(d_lsp, d_conv, d_cc, a, b, (uint32_t)n, f->lf);
    f->ctx->count();
    FPG_CHECK_LAUNCH();
    f->ready = true;
    return FPG_OK;
}

// ============================================================================
// C ABI: the step
// ============================================================================

extern "C" void fpg_step_params_default(fpg_step_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->stages = FPG_STAGE_ALL;
    p->alpha = 0.0f;
    p->dt_seconds = 1.0f;
    p->turb_dt_seconds = 1.0f;
    p->x_grid_per_meter = 1.0f;
    p->y_grid_per_meter = 1.0f;
    p->z_grid_per_meter = 1.0f;
    p->n_substeps = 4;
    p->min_height_m = 0.01f;
    p->dry_reference_height_m = 15.0f;
    p->dry_mode = FPG_FORCING_NONE;
    p->wet_mode = FPG_FORCING_NONE;
}

static void counter_add64(const uint32_t in[4], uint64_t off, uint32_t out[4]) {
    // philox_counter_add (rng.rs:69-87)
    const uint32_t lo = (uint32_t)off, hi = (uint32_t)(off >> 32);
    uint32_t c0 = in[0] + lo;
    uint32_t carry0 = c0 < in[0];
    uint32_t n1 = in[1] + hi;
    uint32_t carry1a = n1 < in[1];
    uint32_t c1 = n1 + carry0;
    uint32_t carry1b = c1 < n1;
    uint32_t c2 = in[2] + (carry1a | carry1b);
    uint32_t carry2 = c2 < in[2];
    uint32_t c3 = in[3] + carry2;
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

extern "C" fpg_status fpg_step(fpg_ctx* ctx, fpg_particles* P, const fpg_met* met, const fpg_pbl* pbl,
                               const fpg_step_params* prm, uint32_t next_counter[4], void* stream) {
    if (!ctx || !P || !prm) return FPG_ERR_INVALID_ARGUMENT;
    if (next_counter) std::memcpy(next_counter, prm->counter, sizeof(uint32_t) * 4);
    const size_t n = P->dispatch;
    if (n == 0) return FPG_OK;                          // empty set: Ok, counter unchanged
    if (n > (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    const uint32_t st = prm->stages & FPG_STAGE_ALL;
    const bool adv = st & FPG_STAGE_ADVECT, turb = st & FPG_STAGE_TURBULENCE;
    const bool dry = (st & FPG_STAGE_DRY) && prm->dry_mode != FPG_FORCING_NONE;
    const bool wet = (st & FPG_STAGE_WET) && prm->wet_mode != FPG_FORCING_NONE;
    if (adv) {
        if (!met) return FPG_ERR_INVALID_ARGUMENT;
        if (!met->uploaded[0] || !met->uploaded[1]) return FPG_ERR_NOT_READY;
        if (!std::isfinite(prm->dt_seconds)) return FPG_ERR_INVALID_TIME_STEP;   // gpu/advection.rs:618
    }
    if (turb) {
        if (!pbl) return FPG_ERR_INVALID_ARGUMENT;
        if (!pbl->ready) return FPG_ERR_NOT_READY;
        if (!std::isfinite(prm->turb_dt_seconds) || prm->turb_dt_seconds <= 0.0f)
            return FPG_ERR_INVALID_TIME_STEP;                                      // langevin_fused.rs:147
    }
    if (dry) {
        if (prm->dry_mode < FPG_FORCING_UNIFORM || prm->dry_mode > FPG_FORCING_PER_PARTICLE)
            return FPG_ERR_INVALID_ARGUMENT;
        if (prm->dry_mode == FPG_FORCING_PER_PARTICLE && !prm->dry_velocity_dev) return FPG_ERR_INVALID_ARGUMENT;
        if (!std::isfinite(prm->turb_dt_seconds)) return FPG_ERR_INVALID_TIME_STEP;  // deposition.rs:334
        if (!std::isfinite(prm->dry_reference_height_m) || prm->dry_reference_height_m <= 0.0f)
            return FPG_ERR_INVALID_REFERENCE_HEIGHT;                                 // deposition.rs:339
    }
    if (wet) {
        if (prm->wet_mode < FPG_FORCING_UNIFORM || prm->wet_mode > FPG_FORCING_PER_CELL)
            return FPG_ERR_INVALID_ARGUMENT;
        if (prm->wet_mode == FPG_FORCING_PER_PARTICLE && (!prm->wet_lambda_dev || !prm->wet_fraction_dev))
            return FPG_ERR_INVALID_ARGUMENT;
        if (prm->wet_mode == FPG_FORCING_PER_CELL && (!prm->wet_cells || !prm->wet_cells->ready))
            return FPG_ERR_NOT_READY;
        if (!std::isfinite(prm->turb_dt_seconds)) return FPG_ERR_INVALID_TIME_STEP;  // wet_deposition.rs:387
    }

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
    a.n = (uint32_t)n;
    a.n_species = P->n_species;
    a.stages = (adv ? FPG_STAGE_ADVECT : 0u) | (turb ? FPG_STAGE_TURBULENCE : 0u) | (dry ? FPG_STAGE_DRY : 0u) |
               (wet ? FPG_STAGE_WET : 0u);
    size_t smem = 0;
    if (adv) {
        a.bracket = met->bracket;
        a.nx = (uint32_t)met->nx; a.ny = (uint32_t)met->ny; a.nz = (uint32_t)met->nz;
        a.has_heights = met->heights_set && met->heights[met->nz - 1] > 0.0f;
        a.level_mode = level_mode(met);
        a.level_table = met->level_table_dev;
        a.level_inv_w = met->level_inv_w;
        // gpu/advection.rs:639: alpha clamped to [0, 1]
        a.alpha = fminf(fmaxf(prm->alpha, 0.0f), 1.0f);
        a.dt = prm->dt_seconds;
        a.xs = prm->x_grid_per_meter; a.ys = prm->y_grid_per_meter; a.zs = prm->z_grid_per_meter;
        smem = level_smem_bytes(met);
        a.heights = met->heights_dev;
    }
    if (turb) {
        a.hcell = pbl->hanna;
        a.pnx = (uint32_t)pbl->nx; a.pny = (uint32_t)pbl->ny;
        a.tdt = prm->turb_dt_seconds;
        a.rho = prm->rho_grad_over_rho;
        a.zmin = prm->min_height_m;
        a.n_sub = prm->n_substeps;
        a.key0 = prm->key[0]; a.key1 = prm->key[1];
        a.counter = u32x4{prm->counter[0], prm->counter[1], prm->counter[2], prm->counter[3]};
    } else {
        a.tdt = prm->turb_dt_seconds;
    }
    a.href = fmaxf(prm->dry_reference_height_m, 0.1f);                // dry_deposition.wgsl:89
    a.dry_mode = dry ? prm->dry_mode : FPG_FORCING_NONE;
    a.dry_v = prm->dry_velocity_m_s;
    a.dry_v_arr = prm->dry_velocity_dev;
    a.dry_prob = prm->dry_probability_dev;
    a.wet_mode = wet ? prm->wet_mode : FPG_FORCING_NONE;
    a.wet_l = prm->wet_lambda_s_inv;
    a.wet_f = prm->wet_fraction;
    a.wet_l_arr = prm->wet_lambda_dev;
    a.wet_f_arr = prm->wet_fraction_dev;
    if (wet && prm->wet_mode == FPG_FORCING_PER_CELL) {
        a.wet_cells = prm->wet_cells->lf;
        a.wnx = (uint32_t)prm->wet_cells->nx; a.wny = (uint32_t)prm->wet_cells->ny;
    }
    a.wet_prob = prm->wet_probability_dev;

    cudaStream_t s = ctx->pick(stream);
    const StepShape& sh = kStepShapes[ctx->step_shape < kNumStepShapes ? ctx->step_shape : 0];
    sh.kernel<<<blocks_for(n, sh.block * sh.ppt), sh.block, sh.ppt > 1 ? smem : 0, s>>>(a);
    ctx->count();
    FPG_CHECK_LAUNCH();
    if (turb && next_counter) {
        // gpu/langevin_fused.rs:229-233
        const uint64_t bpp = prm->n_substeps <= 2u ? 1u : 2u;
        counter_add64(prm->counter, (uint64_t)n * bpp, next_counter);
    }
    return FPG_OK;
}

namespace fpg {
size_t particles_block_bytes(size_t capacity);
}

extern "C" uint32_t fpg_step_tuning_candidates(fpg_batch_tuning* out, uint32_t max) {
    for (uint32_t v = 0; out && v < kNumStepShapes && v < max; ++v)
        out[v] = fpg_batch_tuning{kStepShapes[v].block, kStepShapes[v].minb, kStepShapes[v].ppt, 0.0f};
    return kNumStepShapes;
}

extern "C" fpg_status fpg_step_set_tuning(fpg_ctx* ctx, const fpg_batch_tuning* t) {
    if (!ctx || !t) return FPG_ERR_INVALID_ARGUMENT;
    for (uint32_t v = 0; v < kNumStepShapes; ++v)
        if (kStepShapes[v].block == t->block_threads && kStepShapes[v].minb == t->min_blocks_per_sm &&
            kStepShapes[v].ppt == t->particles_per_thread) {
            ctx->step_shape = v;
            return FPG_OK;
        }
    return FPG_ERR_INVALID_ARGUMENT;
}

extern "C" fpg_status fpg_step_get_tuning(const fpg_ctx* ctx, fpg_batch_tuning* t) {
    if (!ctx || !t) return FPG_ERR_INVALID_ARGUMENT;
    const StepShape& sh = kStepShapes[ctx->step_shape < kNumStepShapes ? ctx->step_shape : 0];
    *t = fpg_batch_tuning{sh.block, sh.minb, sh.ppt, 0.0f};
    return FPG_OK;
}

// auto_tune_key_kernels (src/gpu/workgroup.rs:377-440) for the fused step:
// every compiled shape timed from one snapshot of the particle arrays (the
// restore copy also evicts them from L2), fastest kept.
extern "C" fpg_status fpg_step_autotune(fpg_ctx* ctx, fpg_particles* P, const fpg_met* met, const fpg_pbl* pbl,
                                        const fpg_step_params* prm, uint32_t reps, fpg_batch_tuning* results,
                                        uint32_t max_results, fpg_batch_tuning* best, void* stream) {
    if (!ctx || !P || !prm) return FPG_ERR_INVALID_ARGUMENT;
    if (reps == 0) reps = 1;
    cudaStream_t s = ctx->pick(stream);
    const size_t bytes = particles_block_bytes(P->capacity);
    const uint32_t keep = ctx->step_shape;
    void* snap = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    fpg_status status = FPG_OK;
    uint32_t best_v = keep < kNumStepShapes ? keep : 0;
    float best_ms = 0.0f;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMalloc(&snap, bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(snap, P->block, bytes, cudaMemcpyDeviceToDevice, s);
    for (uint32_t v = 0; e == cudaSuccess && status == FPG_OK && v < kNumStepShapes; ++v) {
        ctx->step_shape = v;
        float tmin = 0.0f;
        for (uint32_t r = 0; r < reps; ++r) {
            e = cudaMemcpyAsync(P->block, snap, bytes, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(e0, s);
            if (e != cudaSuccess) break;
            status = fpg_step(ctx, P, met, pbl, prm, nullptr, s);
            if (status != FPG_OK) break;
            e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) break;
            if (r == 0 || ms < tmin) tmin = ms;
        }
        if (e != cudaSuccess || status != FPG_OK) break;
        if (results && v < max_results)
            results[v] = fpg_batch_tuning{kStepShapes[v].block, kStepShapes[v].minb, kStepShapes[v].ppt, tmin};
        if (v == 0 || tmin < best_ms) { best_ms = tmin; best_v = v; }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(P->block, snap, bytes, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(snap);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e != cudaSuccess || status != FPG_OK) {
        ctx->step_shape = keep;
        return e != cudaSuccess ? cuda_status(e) : status;
    }
    ctx->step_shape = best_v;
    if (best) *best = fpg_batch_tuning{kStepShapes[best_v].block, kStepShapes[best_v].minb, kStepShapes[best_v].ppt,
                                       best_ms};
    return FPG_OK;
}

extern "C" fpg_status fpg_advect_dual_wind(fpg_ctx* ctx, fpg_particles* particles, const fpg_met* met, float alpha,
                                           float dt_seconds, float xs, float ys, float zs, void* stream) {
    fpg_step_params p;
    fpg_step_params_default(&p);
    p.stages = FPG_STAGE_ADVECT;
    p.alpha = alpha;
    p.dt_seconds = dt_seconds;
    p.x_grid_per_meter = xs; p.y_grid_per_meter = ys; p.z_grid_per_meter = zs;
    return fpg_step(ctx, particles, met, nullptr, &p, nullptr, stream);
}

extern "C" fpg_status fpg_langevin_fused(fpg_ctx* ctx, fpg_particles* particles, const fpg_pbl* pbl, float dt,
                                         float rho_grad_over_rho, uint32_t n_substeps, float min_height_m,
                                         const uint32_t key[2], const uint32_t base_counter[4],
                                         uint32_t next_counter[4], void* stream) {
    if (!key || !base_counter) return FPG_ERR_INVALID_ARGUMENT;
    fpg_step_params p;
    fpg_step_params_default(&p);
    p.stages = FPG_STAGE_TURBULENCE;
    p.turb_dt_seconds = dt;
    p.rho_grad_over_rho = rho_grad_over_rho;
    p.n_substeps = n_substeps;
    p.min_height_m = min_height_m;
    p.key[0] = key[0]; p.key[1] = key[1];
    std::memcpy(p.counter, base_counter, sizeof(p.counter));
    return fpg_step(ctx, particles, nullptr, pbl, &p, next_counter, stream);
}

namespace fpg {
namespace {

struct RecordTurbArgs {
    float* pos_z;
    float* turb_u;
    float* turb_v;
    float* turb_w;
    int32_t* cbt;
    const uint32_t* flags;
    const fpg_hanna_params* hanna;
    uint32_t n;
    float tdt, rho, zmin;
    uint32_t n_sub;
    u32x4 counter;
    uint32_t key0, key1;
};

// hanna_params.wgsl:231-258 with compute_hanna (physics/hanna.rs:49-163):
// one 64-byte HannaParams record per slot, zeros for inactive slots.
// compute_hanna at the slot's height from its cell's Hanna constants (the
// record the PBL pass builds from the same u*, w*, h and 1/L, with the same
// operations as compute_hanna would, so the results are the same bits).
__global__ void __launch_bounds__(256) hanna_params_kernel(SlotView v, const CellHanna* __restrict__ hcell,
                                                           uint32_t pnx, uint32_t pny,
                                                           fpg_hanna_params* __restrict__ out) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= v.n) return;
    float4* o = reinterpret_cast<float4*>(out + p);
    if ((v.flags[p] & FLAG_ACTIVE) == 0u) {
        const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        o[0] = z; o[1] = z; o[2] = z; o[3] = z;
        return;
    }
    const CellHanna cell = ld_cell_hanna(hcell + pbl_cell_index(v, p, pnx, pny));
    const float z = v.pos_z[p];
    const Hanna hn = compute_hanna_cell_t<float>(cell, z);
    // zeta and d(sigma_w^2)/dz as the CPU routine forms them (hanna.rs:55,145)
    const float zeta = clampf(clampf(z, 0.0f, hn.h) / hn.h, 0.0f, 1.0f);
    o[0] = make_float4(hn.ust, hn.wst, hn.ol, hn.h);
    o[1] = make_float4(zeta, hn.sigu, hn.sigv, hn.sigw);
    o[2] = make_float4(hn.dsigwdz, 2.0f * hn.sigw * hn.dsigwdz, hn.tlu, hn.tlv);
    o[3] = make_float4(hn.tlw, 0.0f, 0.0f, 0.0f);
}

// langevin.wgsl:307-424: the turbulence update from a HannaParams record per
// slot (the separated Hanna -> Langevin path of the reference's validation
// and backward loops), with the fused kernel's Philox block layout and
// Gaussian assignment.
__global__ void __launch_bounds__(256) langevin_record_kernel(RecordTurbArgs a) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n || !(a.flags[p] & FLAG_ACTIVE)) return;
    const uint32_t n_vert = a.n_sub > 1u ? a.n_sub : 1u;
    const uint32_t blocks = (2u + n_vert + 3u) / 4u;
    const u32x4 b0 = philox4x32_10(counter_add(a.counter, p * blocks), a.key0, a.key1);
    u32x4 b1 = {0u, 0u, 0u, 0u};
    if (blocks > 1u) b1 = philox4x32_10(counter_add(a.counter, p * blocks + 1u), a.key0, a.key1);
    const float2 e_uv = box_muller(u32_to_uniform01(b0.x), u32_to_uniform01(b0.y));
    const float2 e_w01 = box_muller(u32_to_uniform01(b0.z), u32_to_uniform01(b0.w));
    const float2 e_w23 = box_muller(u32_to_uniform01(b1.x), u32_to_uniform01(b1.y));
    const fpg_hanna_params& r = a.hanna[p];
    Hanna hn;
    hn.ust = r.ust; hn.wst = r.wst; hn.ol = r.ol; hn.h = r.h;
    hn.sigu = r.sigu; hn.sigv = r.sigv; hn.sigw = r.sigw; hn.dsigwdz = r.dsigwdz;
    hn.tlu = r.tlu; hn.tlv = r.tlv; hn.tlw = r.tlw;
    // the vertical re-evaluation's constants; its branch is hanna_short_w's
    // test on (L, max(h, 1))
    const CellHanna cell = cell_hanna(r.ust, r.wst, r.ol, r.h);
    hn.regime = cell.regime;
    float pz = a.pos_z[p], tu = a.turb_u[p], tv = a.turb_v[p], tw = a.turb_w[p];
    const int32_t cbt_in = a.n_sub == 0u ? 0 : a.cbt[p];
    int32_t cbt = cbt_in;
    turbulence_from_hanna<float, RecordLangevin>(a, cell, hn, e_uv, e_w01, e_w23, pz, tu, tv, tw, cbt);
    a.turb_u[p] = tu; a.turb_v[p] = tv; a.turb_w[p] = tw;
    if (a.n_sub != 0u) {
        a.pos_z[p] = pz;
        if (cbt != cbt_in) a.cbt[p] = cbt;
    }
}

}  // namespace
}  // namespace fpg

extern "C" fpg_status fpg_langevin_with_hanna(fpg_ctx* ctx, fpg_particles* P, const fpg_hanna_params* hanna_dev,
                                              size_t n_hanna, float dt, float rho_grad_over_rho, uint32_t n_substeps,
                                              float min_height_m, const uint32_t key[2],
                                              const uint32_t base_counter[4], uint32_t next_counter[4],
                                              void* stream) {
    if (!ctx || !P || !key || !base_counter) return FPG_ERR_INVALID_ARGUMENT;
    const size_t n = P->dispatch;
    if (next_counter) std::memcpy(next_counter, base_counter, sizeof(uint32_t) * 4);
    // encode_update_particles_turbulence_langevin_gpu_with_hanna_buffer_and_kernel
    // (src/gpu/langevin.rs:248-329): MismatchedInputLengths, empty, InvalidTimeStep
    if (n_hanna != n) return FPG_ERR_LENGTH_MISMATCH;
    if (n == 0) return FPG_OK;
    if (!std::isfinite(dt) || dt <= 0.0f) return FPG_ERR_INVALID_TIME_STEP;
    if (n > (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    if (!hanna_dev) return FPG_ERR_INVALID_ARGUMENT;
    RecordTurbArgs a{};
    a.pos_z = static_cast<float*>(P->field[FPG_FIELD_POS_Z]);
    a.turb_u = static_cast<float*>(P->field[FPG_FIELD_TURB_U]);
    a.turb_v = static_cast<float*>(P->field[FPG_FIELD_TURB_V]);
    a.turb_w = static_cast<float*>(P->field[FPG_FIELD_TURB_W]);
    a.cbt = static_cast<int32_t*>(P->field[FPG_FIELD_CBT]);
    a.flags = static_cast<const uint32_t*>(P->field[FPG_FIELD_FLAGS]);
    a.hanna = hanna_dev;
    a.n = (uint32_t)n;
    a.tdt = dt;
    a.rho = rho_grad_over_rho;
    a.zmin = min_height_m;
    a.n_sub = n_substeps;
    a.counter = u32x4{base_counter[0], base_counter[1], base_counter[2], base_counter[3]};
    a.key0 = key[0];
    a.key1 = key[1];
    langevin_record_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->pick(stream)>>>(a);
    ctx->count();
    FPG_CHECK_LAUNCH();
    if (next_counter) counter_add64(base_counter, (uint64_t)n * (n_substeps <= 2u ? 1u : 2u), next_counter);
    return FPG_OK;
}

extern "C" fpg_status fpg_dispatch_hanna_params(fpg_ctx* ctx, const fpg_particles* P, const fpg_pbl* pbl,
                                                fpg_hanna_params* out_dev, size_t n_out, void* stream) {
    if (!ctx || !P || !pbl) return FPG_ERR_INVALID_ARGUMENT;
    if (P->dispatch == 0) return FPG_OK;
    if (n_out != P->dispatch) return FPG_ERR_LENGTH_MISMATCH;
    if (!out_dev || !aligned16(out_dev)) return FPG_ERR_INVALID_ARGUMENT;
    if (pbl->nx == 0 || pbl->ny == 0) return FPG_ERR_ZERO_SHAPE;
    if (pbl->nx > UINT32_MAX || pbl->ny > UINT32_MAX || P->dispatch > UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    if (!pbl->ready) return FPG_ERR_NOT_READY;
    const SlotView v = slot_view(P);
    if (v.n == 0) return FPG_OK;
    hanna_params_kernel<<<(unsigned)((v.n + 255) / 256), 256, 0, ctx->pick(stream)>>>(
        v, pbl->hanna, (uint32_t)pbl->nx, (uint32_t)pbl->ny, out_dev);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}

extern "C" fpg_status fpg_dry_deposition(fpg_ctx* ctx, fpg_particles* particles, const float* vdep_dev, float dt,
                                         float href, float* prob_dev, void* stream) {
    if (!vdep_dev) return FPG_ERR_INVALID_ARGUMENT;
    fpg_step_params p;
    fpg_step_params_default(&p);
    p.stages = FPG_STAGE_DRY;
    p.turb_dt_seconds = dt;
    p.dry_reference_height_m = href;
    p.dry_mode = FPG_FORCING_PER_PARTICLE;
    p.dry_velocity_dev = vdep_dev;
    p.dry_probability_dev = prob_dev;
    return fpg_step(ctx, particles, nullptr, nullptr, &p, nullptr, stream);
}

extern "C" fpg_status fpg_wet_deposition(fpg_ctx* ctx, fpg_particles* particles, const float* lambda_dev,
                                         const float* fraction_dev, float dt, float* prob_dev, void* stream) {
    if (!lambda_dev || !fraction_dev) return FPG_ERR_INVALID_ARGUMENT;
    fpg_step_params p;
    fpg_step_params_default(&p);
    p.stages = FPG_STAGE_WET;
    p.turb_dt_seconds = dt;
    p.wet_mode = FPG_FORCING_PER_PARTICLE;
    p.wet_lambda_dev = lambda_dev;
    p.wet_fraction_dev = fraction_dev;
    p.wet_probability_dev = prob_dev;
    return fpg_step(ctx, particles, nullptr, nullptr, &p, nullptr, stream);
}

extern "C" fpg_status fpg_philox_uniforms(fpg_ctx* ctx, const uint32_t key[2], const uint32_t counter[4],
                                          size_t n_blocks, float* out_dev, uint32_t* raw_dev, void* stream) {
    if (!ctx || !key || !counter) return FPG_ERR_INVALID_ARGUMENT;
    if (n_blocks == 0) return FPG_OK;
    if (n_blocks > (size_t)UINT32_MAX / 4) return FPG_ERR_VALUE_TOO_LARGE;
    cudaStream_t s = ctx->pick(stream);
    philox_kernel<<<blocks_for(n_blocks, 256), 256, 0, s>>>(key[0], key[1],
                                                             u32x4{counter[0], counter[1], counter[2], counter[3]},
                                                             (uint32_t)n_blocks, out_dev, raw_dev);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}
