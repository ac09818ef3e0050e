// cbl.cu — convective-boundary-layer sampling and convective mixing
// (the per-slot Hanna records they read come from fpg_dispatch_hanna_params,
// built with the step in step.cu):
//
// * fpg_cbl_sample: the bi-Gaussian vertical-velocity PDF of the CBL and one
//   sampled w' per slot from caller uniforms (cbl.wgsl, src/gpu/cbl.rs);
// * fpg_cbl_sample_philox: the same sample fused with the Hanna sigma_w at
//   the particle's cell and Philox uniforms, so the per-slot 64-byte Hanna
//   record and the 16-byte uniform record never go through HBM;
// * fpg_convection_*: the column redistribution matrix applied to particle
//   heights (convective_mixing.wgsl, src/gpu/convection.rs).  The expected
//   destination height depends only on the source level, so it is computed
//   once per level when the matrix is set (one thread per level, the same
//   sequential f32 sum the reference runs per particle); the per-particle
//   kernel is a level search plus one table read: 8 bytes read and 8 bytes
//   written per active slot, four slots per thread, HBM-bound.
//
// The PDF follows the CPU routine (physics/cbl.rs:126-226): cbrt for the
// signed cube root and repeated multiplication for powi(3) / powi(2); the
// shader's pow() forms agree within the 5e-5 relative tolerance its own GPU
// test allows (src/gpu/cbl.rs:446-515).
#include <cmath>
#include <cstring>
#include <vector>

#include "fpg_internal.h"
#include "physics.cuh"
#include "slots.cuh"

namespace fpg {
namespace {

constexpr float kMinH = 1.0f;
constexpr float kMinSigmaW = 1.0e-5f;
constexpr float kSkewEps = 1.0e-6f;
constexpr float kW3Eps = 1.0e-6f;
constexpr float kFluarw = 2.0f / 3.0f;
constexpr float kPi = 3.14159265358979323846f;   // std::f32::consts::PI

// cbl_transition_factor (physics/cbl.rs:109-124, cbl.wgsl:133-146).
__device__ __forceinline__ float cbl_transition(float h, float ol) {
    if (!finitef(h) || h <= 0.0f || !finitef(ol) || ol == 0.0f) return 1.0f;
    const float ratio = -h / ol;
    const float t = ratio < 15.0f ? sinf(((ratio + 10.0f) / 10.0f) * kPi) * 0.5f + 0.5f : 1.0f;
    return clampf(t, 0.0f, 1.0f);
}

// CblSamplingOutput field order (src/gpu/cbl.rs:66-92) minus the sample.
struct CblPdf {
    float aw, am, as, bw, bm, bs, w2, w3, skew, trans, zoh;
};

// compute_cbl_moments + compute_cbl_bigaussian_pdf (physics/cbl.rs:126-226).
__device__ __forceinline__ CblPdf cbl_pdf(float z_in, float h_in, float wst_in, float sigw_in, float ol) {
    const float h = fmaxf(h_in, kMinH);
    const float z = clampf(z_in, 0.0f, h);
    const float zoh = z / h;
    const float wst = fmaxf(wst_in, 0.0f);
    const float sw = fmaxf(sigw_in, kMinSigmaW);
    const float trans = cbl_transition(h, ol);
    const float w2 = sw * sw;
    const float shape = 1.2f * zoh * powf(1.0f - zoh, 1.5f) + kW3Eps;
    const float w3 = shape * (wst * wst * wst) * trans;
    const float skew = w3 / powf(w2, 1.5f);
    CblPdf p{0.5f, 0.0f, sw, 0.5f, 0.0f, sw, w2, w3, skew, trans, zoh};
    if (!finitef(skew) || fabsf(skew) <= kSkewEps) return p;
    const float fl = kFluarw * cbrtf(skew);
    const float fl2 = fl * fl;
    if (!finitef(fl) || fabsf(fl) <= kSkewEps) return p;
    const float skew2 = skew * skew;
    const float a1 = 1.0f + fl2, a3 = 3.0f + fl2;
    const float num = (a1 * a1 * a1) * skew2;
    const float den = (a3 * a3) * fl2;
    const float r = fmaxf(num / fmaxf(den, kSkewEps), 0.0f);
    const float x = sqrtf(r);
    const float aw = clampf(0.5f * (1.0f - x / sqrtf(4.0f + r)), 1.0e-4f, 1.0f - 1.0e-4f);
    const float bw = 1.0f - aw;
    const float sa = sw * sqrtf(bw / (aw * (1.0f + fl2)));
    const float sb = sw * sqrtf(aw / (bw * (1.0f + fl2)));
    p.aw = aw; p.am = fl * sa; p.as = fmaxf(sa, kMinSigmaW);
    p.bw = bw; p.bm = -(fl * sb); p.bs = fmaxf(sb, kMinSigmaW);
    return p;
}

// sample_cbl_vertical_velocity (physics/cbl.rs:274-288, cbl.wgsl:270-277).
__device__ __forceinline__ float cbl_draw(const CblPdf& p, float ub, float u0, float u1) {
    const float eta = box_muller(u0, u1).x;
    return ub < p.aw ? p.am + p.as * eta : p.bm + p.bs * eta;
}

__device__ __forceinline__ void store_output(fpg_cbl_sampling_output* out, size_t i, float w, const CblPdf& p) {
    float4* o = reinterpret_cast<float4*>(out + i);
    o[0] = make_float4(w, p.aw, p.am, p.as);
    o[1] = make_float4(p.bw, p.bm, p.bs, p.w2);
    o[2] = make_float4(p.w3, p.skew, p.trans, p.zoh);
}

__device__ __forceinline__ void store_zero_output(fpg_cbl_sampling_output* out, size_t i) {
    float4* o = reinterpret_cast<float4*>(out + i);
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    o[0] = z; o[1] = z; o[2] = z;
}

// cbl.wgsl:251-298: PDF from the slot's Hanna record, sample from its uniforms.
__global__ void __launch_bounds__(256) cbl_sample_kernel(SlotView v, const fpg_hanna_params* __restrict__ hanna,
                                                         const fpg_cbl_sampling_input* __restrict__ in,
                                                         fpg_cbl_sampling_output* __restrict__ out) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= v.n) return;
    if ((v.flags[p] & FLAG_ACTIVE) == 0u) {
        store_zero_output(out, p);
        return;
    }
    const float4 h0 = __ldg(reinterpret_cast<const float4*>(hanna + p));       // ust, wst, ol, h
    const float sigw = __ldg(&hanna[p].sigw);
    const float4 u = __ldg(reinterpret_cast<const float4*>(in + p));
    const CblPdf pdf = cbl_pdf(v.pos_z[p], h0.w, h0.y, sigw, h0.z);
    store_output(out, p, cbl_draw(pdf, u.x, u.y, u.z), pdf);
}

// The fused form: sigma_w of compute_hanna at the slot's cell (the vertical
// branch of hanna_short_w gives the same sigma_w bits as compute_hanna) from
// the cell's Hanna constants (the floored u*, w*, h, the Obukhov length, the
// regime and the constant products the PBL pass stores per cell, so the
// per-cell part is not redone per slot), and the uniforms of one Philox
// block at counter + slot: u0, u1, u2 of PhiloxRng::next_uniform4 on a
// stream that starts at that counter (physics/cbl.rs:291-295,
// physics/rng.rs:130-164).
__global__ void __launch_bounds__(256) cbl_sample_philox_kernel(SlotView v, const CellHanna* __restrict__ hcell,
                                                                uint32_t pnx, uint32_t pny, uint32_t k0,
                                                                uint32_t k1, u32x4 counter,
                                                                fpg_cbl_sampling_output* __restrict__ out) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= v.n) return;
    if ((v.flags[p] & FLAG_ACTIVE) == 0u) {
        store_zero_output(out, p);
        return;
    }
    const CellHanna cell = ld_cell_hanna(hcell + pbl_cell_index(v, p, pnx, pny));
    const float z = v.pos_z[p];
    float sigw, dsigwdz, tlw;
    hanna_short_cell_t<float>(cell, z, sigw, dsigwdz, tlw);
    const u32x4 b = philox4x32_10(counter_add(counter, (uint32_t)p), k0, k1);
    const CblPdf pdf = cbl_pdf(z, cell.h, cell.wst, sigw, cell.ol);
    store_output(out, p, cbl_draw(pdf, u32_to_uniform01(b.x), u32_to_uniform01(b.y), u32_to_uniform01(b.z)), pdf);
}

// expected_destination_height_m (physics/convection.rs:398-427): one thread
// per source level sums its matrix column in destination order, as the
// shader's per-particle loop does (convective_mixing.wgsl:98-104), then
// clamps to the column (the shader's clamp of the quotient).
__global__ void conv_heights_kernel(uint32_t L, const float* __restrict__ m, const float* __restrict__ centers,
                                    float z_min, float z_max, float* __restrict__ heights,
                                    uint32_t* __restrict__ has_weight) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= L) return;
    float wh = 0.0f, ws = 0.0f;
    const float* col = m + (size_t)s * L;
    for (uint32_t d = 0; d < L; ++d) {
        const float w = fmaxf(col[d], 0.0f);
        wh = wh + w * centers[d];
        ws = ws + w;
    }
    has_weight[s] = ws > 0.0f ? 1u : 0u;
    heights[s] = ws > 0.0f ? clampf(wh / ws, z_min, z_max) : 0.0f;
}

// convective_mixing.wgsl:87-113 per active slot.  With strictly increasing
// finite interfaces the shader's linear scan (first level with
// lower <= z < upper, else the top level) is the last level whose lower
// interface is <= z, found by bisection; otherwise the scan itself runs.
template <bool kSorted>
__device__ __forceinline__ uint32_t source_level(float z, uint32_t L, const float* __restrict__ iface) {
    if constexpr (kSorted) {
        uint32_t lo = 0u, hi = L;                 // count of iface[0..L) <= z lies in [1, L]
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(iface + mid) <= z) lo = mid; else hi = mid;
        }
        return lo;
    } else {
        for (uint32_t l = 0; l < L; ++l)
            if (z >= __ldg(iface + l) && z < __ldg(iface + l + 1u)) return l;
        return L - 1u;
    }
}

// The mixed height and the source level of one active slot.
template <bool kSorted>
__device__ __forceinline__ float mix_height(float z_in, uint32_t L, const float* __restrict__ iface,
                                            const float* __restrict__ heights,
                                            const uint32_t* __restrict__ has_weight, float z_min, float z_max,
                                            int32_t& level_out) {
    const float z = clampf(z_in, z_min, z_max);
    const uint32_t level = source_level<kSorted>(z, L, iface);
    level_out = (int32_t)level;
    return __ldg(has_weight + level) ? __ldg(heights + level) : z;
}

template <bool kSorted>
__device__ __forceinline__ void mix_slot(size_t p, float z_in, float* __restrict__ pos_z, int32_t* __restrict__ cbt,
                                         uint32_t L, const float* __restrict__ iface,
                                         const float* __restrict__ heights, const uint32_t* __restrict__ has_weight,
                                         float z_min, float z_max) {
    int32_t level;
    pos_z[p] = mix_height<kSorted>(z_in, L, iface, heights, has_weight, z_min, z_max, level);
    cbt[p] = level;
}

// Four slots per thread: the flags and heights of a quad arrive in one
// 16-byte load each (the fields are 256-byte aligned); a quad of active
// slots is written with one 16-byte store per field, otherwise only the
// active slots are written.  The last n % 4 slots take scalar loads.
template <bool kSorted>
__global__ void __launch_bounds__(256) conv_apply_kernel(size_t n, const uint32_t* __restrict__ flags,
                                                         float* __restrict__ pos_z, int32_t* __restrict__ cbt,
                                                         uint32_t L, const float* __restrict__ iface,
                                                         const float* __restrict__ heights,
                                                         const uint32_t* __restrict__ has_weight) {
    const size_t p0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 4u;
    if (p0 >= n) return;
    const float z_min = __ldg(iface), z_max = __ldg(iface + L);
    if (p0 + 4u <= n) {
        const uint4 f = __ldg(reinterpret_cast<const uint4*>(flags + p0));
        const float4 z = *reinterpret_cast<const float4*>(pos_z + p0);
        if (f.x & f.y & f.z & f.w & FLAG_ACTIVE) {
            int4 lv;
            float4 zo;
            zo.x = mix_height<kSorted>(z.x, L, iface, heights, has_weight, z_min, z_max, lv.x);
            zo.y = mix_height<kSorted>(z.y, L, iface, heights, has_weight, z_min, z_max, lv.y);
            zo.z = mix_height<kSorted>(z.z, L, iface, heights, has_weight, z_min, z_max, lv.z);
            zo.w = mix_height<kSorted>(z.w, L, iface, heights, has_weight, z_min, z_max, lv.w);
            *reinterpret_cast<float4*>(pos_z + p0) = zo;
            *reinterpret_cast<int4*>(cbt + p0) = lv;
            return;
        }
        if (f.x & FLAG_ACTIVE) mix_slot<kSorted>(p0, z.x, pos_z, cbt, L, iface, heights, has_weight, z_min, z_max);
        if (f.y & FLAG_ACTIVE) mix_slot<kSorted>(p0 + 1, z.y, pos_z, cbt, L, iface, heights, has_weight, z_min, z_max);
        if (f.z & FLAG_ACTIVE) mix_slot<kSorted>(p0 + 2, z.z, pos_z, cbt, L, iface, heights, has_weight, z_min, z_max);
        if (f.w & FLAG_ACTIVE) mix_slot<kSorted>(p0 + 3, z.w, pos_z, cbt, L, iface, heights, has_weight, z_min, z_max);
    } else {
        for (size_t p = p0; p < n; ++p)
            if (flags[p] & FLAG_ACTIVE)
                mix_slot<kSorted>(p, pos_z[p], pos_z, cbt, L, iface, heights, has_weight, z_min, z_max);
    }
}

}  // namespace
}  // namespace fpg

using namespace fpg;

struct fpg_convection {
    fpg_ctx* ctx = nullptr;
    size_t levels = 0;
    float* matrix = nullptr;        // levels^2, column-major (source * levels + destination)
    float* iface = nullptr;         // levels + 1
    float* centers = nullptr;       // levels
    float* heights = nullptr;       // levels: expected destination height per source level
    uint32_t* has_weight = nullptr; // levels
    bool sorted = true;
    bool ready = false;
};

extern "C" fpg_status fpg_cbl_sample(fpg_ctx* ctx, const fpg_particles* P, const fpg_hanna_params* hanna_dev,
                                     size_t n_hanna, const fpg_cbl_sampling_input* inputs_dev, size_t n_inputs,
                                     fpg_cbl_sampling_output* out_dev, void* stream) {
    if (!ctx || !P) return FPG_ERR_INVALID_ARGUMENT;
    const SlotView v = slot_view(P);
    // GpuCblError::MismatchedInputLengths (src/gpu/cbl.rs:210-216)
    if (n_hanna != v.n || n_inputs != v.n) return FPG_ERR_LENGTH_MISMATCH;
    if (v.n == 0) return FPG_OK;
    if (!hanna_dev || !inputs_dev || !out_dev) return FPG_ERR_INVALID_ARGUMENT;
    if (!aligned16(hanna_dev) || !aligned16(inputs_dev) || !aligned16(out_dev)) return FPG_ERR_INVALID_ARGUMENT;
    if (v.n > UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    cbl_sample_kernel<<<(unsigned)((v.n + 255) / 256), 256, 0, ctx->pick(stream)>>>(v, hanna_dev, inputs_dev,
                                                                                   out_dev);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}

extern "C" fpg_status fpg_cbl_sample_philox(fpg_ctx* ctx, const fpg_particles* P, const fpg_pbl* pbl,
                                            const uint32_t key[2], const uint32_t counter[4],
                                            fpg_cbl_sampling_output* out_dev, void* stream) {
    if (!ctx || !P || !pbl || !key || !counter) return FPG_ERR_INVALID_ARGUMENT;
    if (pbl->nx == 0 || pbl->ny == 0) return FPG_ERR_ZERO_SHAPE;
    if (pbl->nx > UINT32_MAX || pbl->ny > UINT32_MAX || P->dispatch > UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    if (!pbl->ready) return FPG_ERR_NOT_READY;
    const SlotView v = slot_view(P);
    if (v.n == 0) return FPG_OK;
    if (!out_dev || !aligned16(out_dev)) return FPG_ERR_INVALID_ARGUMENT;
    const u32x4 c{counter[0], counter[1], counter[2], counter[3]};
    cbl_sample_philox_kernel<<<(unsigned)((v.n + 255) / 256), 256, 0, ctx->pick(stream)>>>(
        v, pbl->hanna, (uint32_t)pbl->nx, (uint32_t)pbl->ny, key[0], key[1], c, out_dev);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}

extern "C" fpg_status fpg_convection_create(fpg_ctx* ctx, size_t level_count, fpg_convection** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    // GpuConvectionError::InvalidLevelCount (src/gpu/convection.rs:74-79)
    if (level_count == 0) return FPG_ERR_ZERO_SHAPE;
    if (level_count > (size_t)INT32_MAX || level_count > (size_t)65535) return FPG_ERR_VALUE_TOO_LARGE;
    auto* c = new fpg_convection;
    c->ctx = ctx;
    c->levels = level_count;
    const size_t L = level_count;
    cudaError_t e = cudaMalloc(&c->matrix, L * L * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->iface, (L + 1) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->centers, L * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->heights, L * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->has_weight, L * sizeof(uint32_t));
    if (e != cudaSuccess) {
        fpg_convection_destroy(c);
        return cuda_status(e);
    }
    *out = c;
    return FPG_OK;
}

extern "C" fpg_status fpg_convection_destroy(fpg_convection* c) {
    if (!c) return FPG_ERR_INVALID_ARGUMENT;
    cudaFree(c->matrix);
    cudaFree(c->iface);
    cudaFree(c->centers);
    cudaFree(c->heights);
    cudaFree(c->has_weight);
    delete c;
    return FPG_OK;
}

extern "C" fpg_status fpg_convection_set_matrix(fpg_convection* c, const float* matrix_column_major,
                                                size_t n_matrix, const float* level_interfaces_m,
                                                size_t n_interfaces, void* stream) {
    if (!c || !matrix_column_major || !level_interfaces_m) return FPG_ERR_INVALID_ARGUMENT;
    const size_t L = c->levels;
    // ConvectionError::MatrixLengthMismatch (physics/convection.rs:163-170) and
    // GpuConvectionError::InvalidLevelInterfaces (src/gpu/convection.rs:81-86)
    if (n_matrix != L * L || n_interfaces != L + 1) return FPG_ERR_LENGTH_MISMATCH;
    // validate_column_stochasticity (physics/convection.rs:196-218): the
    // reference's matrix type holds this invariant from construction.
    for (size_t s = 0; s < L; ++s) {
        float sum = 0.0f;
        for (size_t d = 0; d < L; ++d) {
            const float w = matrix_column_major[s * L + d];
            if (w < -1.0e-4f || !std::isfinite(w)) return FPG_ERR_NON_STOCHASTIC_COLUMN;
            sum += w;
        }
        if (std::fabs(sum - 1.0f) > 1.0e-4f) return FPG_ERR_NON_STOCHASTIC_COLUMN;
    }
    bool sorted = true;
    for (size_t l = 0; l <= L; ++l) {
        if (!std::isfinite(level_interfaces_m[l]) || (l > 0 && !(level_interfaces_m[l] > level_interfaces_m[l - 1])))
            sorted = false;
    }
    // level_centers_from_interfaces (src/gpu/convection.rs:63-69)
    std::vector<float> centers(L);
    for (size_t l = 0; l < L; ++l) centers[l] = 0.5f * (level_interfaces_m[l] + level_interfaces_m[l + 1]);
    cudaStream_t s = c->ctx->pick(stream);
    FPG_CUDA(cudaMemcpyAsync(c->matrix, matrix_column_major, L * L * sizeof(float), cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(c->iface, level_interfaces_m, (L + 1) * sizeof(float), cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemcpyAsync(c->centers, centers.data(), L * sizeof(float), cudaMemcpyHostToDevice, s));
    conv_heights_kernel<<<(unsigned)((L + 127) / 128), 128, 0, s>>>((uint32_t)L, c->matrix, c->centers,
                                                                   level_interfaces_m[0], level_interfaces_m[L],
                                                                   c->heights, c->has_weight);
    c->ctx->count();
    FPG_CHECK_LAUNCH();
    // the host vector is released on return: wait for its copy
    FPG_CUDA(cudaStreamSynchronize(s));
    c->sorted = sorted;
    c->ready = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_convection_heights(const fpg_convection* c, float* heights_host) {
    if (!c || !heights_host) return FPG_ERR_INVALID_ARGUMENT;
    if (!c->ready) return FPG_ERR_NOT_READY;
    FPG_CUDA(cudaMemcpy(heights_host, c->heights, c->levels * sizeof(float), cudaMemcpyDeviceToHost));
    return FPG_OK;
}

extern "C" fpg_status fpg_convective_mixing(fpg_ctx* ctx, fpg_particles* P, const fpg_convection* c, void* stream) {
    if (!ctx || !P || !c) return FPG_ERR_INVALID_ARGUMENT;
    if (!c->ready) return FPG_ERR_NOT_READY;
    const size_t n = P->dispatch;
    if (n == 0) return FPG_OK;
    if (n > UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    const auto* flags = static_cast<const uint32_t*>(P->field[FPG_FIELD_FLAGS]);
    auto* pos_z = static_cast<float*>(P->field[FPG_FIELD_POS_Z]);
    auto* cbt = static_cast<int32_t*>(P->field[FPG_FIELD_CBT]);
    const unsigned grid = (unsigned)(((n + 3) / 4 + 255) / 256);
    if (c->sorted)
        conv_apply_kernel<true><<<grid, 256, 0, ctx->pick(stream)>>>(n, flags, pos_z, cbt, (uint32_t)c->levels,
                                                                    c->iface, c->heights, c->has_weight);
    else
        conv_apply_kernel<false><<<grid, 256, 0, ctx->pick(stream)>>>(n, flags, pos_z, cbt, (uint32_t)c->levels,
                                                                     c->iface, c->heights, c->has_weight);
    ctx->count();
    FPG_CHECK_LAUNCH();
    return FPG_OK;
}
