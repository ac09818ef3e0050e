// adjoint.cu — source inversion on the batched step: receptor sampling, a
// checkpointed forward, a taped recompute of each K-step window and the
// hand-written reverse of the step (include/fpg_adjoint.h).
//
// Per particle the differentiated state is S = (x, y, z, tu, tv, tw, m):
// continuous grid coordinates x = cell_x + pos_x, y likewise, height z [m],
// turbulent velocities and species-0 mass.  One step maps S_k to S_{k+1}:
//   advection   (x, y, z, tu, tv) -> (x1, y1, z1)          (Petterssen, two
//               dual-time trilinear samples s0 at (x, y, z), s1 at the
//               predictor point, each + the wind bias)
//   turbulence  (z1, tu, tv, tw)  -> (z2, tu', tv', tw')   (Hanna at z1,
//               Langevin, vertical sub-steps with reflection)
//   deposition  m -> m * survival                          (survival fixed)
// The tape kernel runs the step with the turbulence block on dual numbers
// (dual.cuh), which gives its 2x2 vertical and per-component horizontal
// Jacobians with values identical to the plain step, and records the
// advection points, clamp states, survival and the output state.  The
// adjoint kernel then adds the receptor term of sampling steps and applies
// the transposed step to the adjoint state lambda, re-gathering the two wind
// samples' corners for their spatial derivatives and scattering
// lambda_sample x trilinear weight into the bias gradient.
//
// The tape is recorded either during the forward itself (checkpoint_every
// == 0: one tape slice per step, no recompute) or, to bound memory, per
// K-step window from checkpoints during the backward.  Tape slices are
// indexed on the device by step % slices, so one captured graph serves
// every step of either mode.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "../../include/fpg_adjoint.h"
#include "batch_core.cuh"
#include "dual.cuh"
#include "fpg_internal.h"

namespace fpg {

enum TapeField {
    T_X0, T_Y0, T_Z0, T_PX, T_PY, T_PZ,          // advection input point and predictor point
    T_ZZ, T_ZTW, T_WZ, T_WTW, T_UZ, T_UU, T_VZ, T_VV,  // turbulence Jacobian
    T_SURV, T_FLAGS,                             // mass survival, clamp bits | TAPE_ACTIVE
    T_X2, T_Y2, T_Z2, T_M2,                      // the step's output state (receptor term)
    TAPE_FIELDS
};
constexpr uint32_t TAPE_ACTIVE = 0x80000000u;

enum LamField { L_X, L_Y, L_Z, L_TU, L_TV, L_TW, L_M, LAM_FIELDS };

// Tape slice j of a step holds TAPE_FIELDS arrays of `cap` floats at
// base + j * TAPE_FIELDS * cap.
struct TapeBase {
    float* base;
    size_t cap;
    uint32_t slices;
    __device__ __forceinline__ float* field(uint32_t j, int f) const {
        return base + ((size_t)j * TAPE_FIELDS + (size_t)f) * cap;
    }
};
struct TapeArrays { float* f[TAPE_FIELDS]; };
struct LamArrays { float* f[LAM_FIELDS]; };

// The receptor model shared by the forward sampling and the seeds.
struct Receptors {
    const int32_t* rmap;     // per instance, nx*ny cells (i*ny + j): receptor index or -1
    uint32_t nx, ny, cells;
    float ztop, ramp;
    uint32_t every;
    const float* g;          // dL/dsim per receptor (backward)
    double* sim;             // forward sums
    uint32_t* last_hit;      // per slot: 1 + the last step whose output state met a receptor cell (0: none)
};

struct Cic {
    int i0, j0;
    float wx[2], wy[2];
    float v, dv;
};

// Cloud-in-cell weights of the cells around (x, y) (centres at i + 0.5) and
// the vertical weight with its slope.
__device__ __forceinline__ Cic cic(const Receptors& r, float x, float y, float z) {
    Cic c;
    const float xs = x - 0.5f, ys = y - 0.5f;
    const float fi = floorf(xs), fj = floorf(ys);
    c.i0 = (int)fi;
    c.j0 = (int)fj;
    c.wx[1] = xs - fi; c.wx[0] = 1.0f - c.wx[1];
    c.wy[1] = ys - fj; c.wy[0] = 1.0f - c.wy[1];
    const float q = (r.ztop + 0.5f * r.ramp - z) / r.ramp;
    c.v = clampf(q, 0.0f, 1.0f);
    c.dv = (q > 0.0f && q < 1.0f) ? -1.0f / r.ramp : 0.0f;
    return c;
}

__device__ __forceinline__ int receptor_at(const Receptors& r, uint32_t inst, int i, int j) {
    if (i < 0 || j < 0 || i >= (int)r.nx || j >= (int)r.ny) return -1;
    return r.rmap[(size_t)inst * r.cells + (uint32_t)i * r.ny + (uint32_t)j];
}

// ---- forward sampling ---------------------------------------------------------

__global__ void __launch_bounds__(256) inverse_sample_kernel(const BatchState* st, const ScenDev* __restrict__ sc,
                                                             const uint2* __restrict__ items, uint32_t n_items,
                                                             PopFields F, Receptors r) {
    if (r.every == 0 || (st->step + 1u) % r.every != 0u) return;
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
        const uint2 w = items[it];
        const ScenDev& d = sc[w.x];
        const uint32_t local = w.y + threadIdx.x;
        if (local >= d.released) continue;
        const uint32_t p = d.offset + local;
        if (!(F.f[FPG_FIELD_FLAGS][p] & 1u)) continue;
        const float x = (float)(int32_t)F.f[FPG_FIELD_CELL_X][p] + __uint_as_float(F.f[FPG_FIELD_POS_X][p]);
        const float y = (float)(int32_t)F.f[FPG_FIELD_CELL_Y][p] + __uint_as_float(F.f[FPG_FIELD_POS_Y][p]);
        const float z = __uint_as_float(F.f[FPG_FIELD_POS_Z][p]);
        const float m = __uint_as_float(F.f[FPG_FIELD_MASS0][p]);
        const Cic c = cic(r, x, y, z);
        if (c.v == 0.0f) continue;
        bool hit = false;
#pragma unroll
        for (int di = 0; di < 2; ++di)
#pragma unroll
            for (int dj = 0; dj < 2; ++dj) {
                const int rr = receptor_at(r, d.instance, c.i0 + di, c.j0 + dj);
                if (rr >= 0) {
                    atomicAdd(r.sim + rr, (double)(m * (c.wx[di] * c.wy[dj] * c.v)));
                    hit = true;
                }
            }
        // every receptor seed of this output state (receptor_seed) comes from
        // these cells, whatever their weights
        if (hit) r.last_hit[p] = st->step + 1u;
    }
}

// ---- taped recompute ------------------------------------------------------------

struct TapeRec {
    static constexpr bool on = true;
    TapeArrays t;
    bool output;   // a sampling step: the output state is read by the reverse
    __device__ __forceinline__ void advect(uint32_t p, float x0, float y0, float z0, float px, float py, float pz,
                                           uint32_t fl) {
        t.f[T_X0][p] = x0; t.f[T_Y0][p] = y0; t.f[T_Z0][p] = z0;
        t.f[T_PX][p] = px; t.f[T_PY][p] = py; t.f[T_PZ][p] = pz;
        reinterpret_cast<uint32_t*>(t.f[T_FLAGS])[p] = fl | TAPE_ACTIVE;
    }
    __device__ __forceinline__ void turb(uint32_t p, float zz, float ztw, float wz, float wtw, float uz, float uu,
                                         float vz, float vv) {
        t.f[T_ZZ][p] = zz; t.f[T_ZTW][p] = ztw; t.f[T_WZ][p] = wz; t.f[T_WTW][p] = wtw;
        t.f[T_UZ][p] = uz; t.f[T_UU][p] = uu; t.f[T_VZ][p] = vz; t.f[T_VV][p] = vv;
    }
    __device__ __forceinline__ void deposit(uint32_t p, float s) { t.f[T_SURV][p] = s; }
    __device__ __forceinline__ void out(uint32_t p, float x, float y, float z, float m) {
        if (output) { t.f[T_X2][p] = x; t.f[T_Y2][p] = y; t.f[T_Z2][p] = z; t.f[T_M2][p] = m; }
    }
};

// Post-advance clock and scenario state of the step, kept per tape slice.
__global__ void inverse_snapshot_kernel(const BatchState* st, const ScenDev* __restrict__ sc, uint32_t n_scen,
                                        uint32_t slices, BatchState* st_all, ScenDev* sc_all) {
    const uint32_t j = st->step % slices;
    if (threadIdx.x == 0 && blockIdx.x == 0) st_all[j] = *st;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_scen; s += gridDim.x * blockDim.x)
        sc_all[(size_t)j * n_scen + s] = sc[s];
}

// `live` (the recompute of a checkpoint window; NULL in the forward): a slot
// whose last receptor hit came before this step has a zero adjoint from this
// step on, so its tape is never read -- it is marked inactive for the
// reverse and not stepped.
// One CTA per 256-slot work item, launched over all items; the level arrays
// are read from global memory (no staging, no barrier).
__global__ void __launch_bounds__(256, 4) inverse_tape_kernel(StepArgs a, const BatchState* st,
                                                              const ScenDev* __restrict__ sc,
                                                              const uint2* __restrict__ items, uint32_t n_items,
                                                              TapeBase tb, uint32_t every,
                                                              const uint32_t* __restrict__ live) {
    if (blockIdx.x >= n_items) return;
    const uint2 w = items[blockIdx.x];
    const ScenDev& d = sc[w.x];
    const uint32_t local = w.y + threadIdx.x;
    if (local >= d.released) return;
    const uint32_t slice = st->step % tb.slices;
    TapeRec rec;
    rec.output = every != 0 && (st->step + 1u) % every == 0u;
#pragma unroll
    for (int f = 0; f < TAPE_FIELDS; ++f) rec.t.f[f] = tb.field(slice, f);
    const uint32_t p = d.offset + local;
    if (!(a.flags[p] & FLAG_ACTIVE) || (live && live[p] <= st->step)) {
        reinterpret_cast<uint32_t*>(rec.t.f[T_FLAGS])[p] = 0u;
        return;
    }
    particle_step_t<TapeRec>(a, global_levels(a), p, local, st->alpha, d.counter, d.key0, d.key1, rec);
}

// ---- reverse ----------------------------------------------------------------------

// meters_to_level with its slope d(level)/dz.
__device__ __forceinline__ float level_slope(const Levels& L, float z) {
    if (!L.has) return 1.0f;
    const float* h = L.h;
    const uint32_t nz = L.nz;
    const float h0 = h[0];
    if (z <= h0) return h0 > 0.0f ? 1.0f / h0 : 0.0f;
    const uint32_t k = level_index(L, z);
    if (k >= nz) return 0.0f;
    const float denom = h[k] - h[k - 1u];
    return denom > 0.0f ? 1.0f / denom : 0.0f;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums each of the 24 values v[0..23] over the 32 lanes with a transposed
// butterfly (12 + 6 + 3 exchanges halve the values a lane holds while
// doubling the lanes summed, then 2 x 3 exchanges finish the 3 left): 27
// shuffles instead of 24 x 5.  On return v[0..2] of every lane hold the
// full sums of values 3c .. 3c+2, c = lane >> 2 (lanes 4c .. 4c+3 agree).
__device__ __forceinline__ void warp_sum24(float (&v)[24], unsigned lane) {
    const bool b4 = lane & 16u, b3 = lane & 8u, b2 = lane & 4u;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const float send = b4 ? v[i] : v[i + 12];
        const float keep = b4 ? v[i + 12] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float send = b3 ? v[i] : v[i + 6];
        const float keep = b3 ? v[i + 6] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float send = b2 ? v[i] : v[i + 3];
        const float keep = b2 ? v[i + 3] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        v[i] += __shfl_xor_sync(0xffffffffu, v[i], 2);
        v[i] += __shfl_xor_sync(0xffffffffu, v[i], 1);
    }
}

// The CTA's table of bias-gradient nodes for one adjoint step: open
// addressing on the node index in shared memory, three float sums per node,
// added to the f64 gradient once per node per CTA at the end of the step.
// The f64 atomics of the per-warp sums were the cost of the whole reverse
// sweep (two thirds of it); the table takes them off the L2.
constexpr uint32_t kBiasTableBits = 10;
constexpr uint32_t kBiasTable = 1u << kBiasTableBits;
constexpr uint32_t kBiasProbes = 8;
constexpr uint32_t kBiasEmpty = 0xffffffffu;

struct BiasTable {
    uint32_t* key;   // kBiasTable
    float* g;        // 3 * kBiasTable
};

__device__ __forceinline__ void bias_add(const BiasTable& t, uint32_t n, float gu, float gv, float gw,
                                         double* __restrict__ dbias) {
    uint32_t slot = (n * 2654435761u) >> (32 - kBiasTableBits);
    for (uint32_t i = 0; i < kBiasProbes; ++i) {
        const uint32_t old = atomicCAS(t.key + slot, kBiasEmpty, n);
        if (old == kBiasEmpty || old == n) {
            atomicAdd(t.g + 3u * slot + 0u, gu);
            atomicAdd(t.g + 3u * slot + 1u, gv);
            atomicAdd(t.g + 3u * slot + 2u, gw);
            return;
        }
        slot = (slot + 1u) & (kBiasTable - 1u);
    }
    atomicAdd(dbias + 3u * n + 0u, (double)gu);     // crowded table: straight to the gradient
    atomicAdd(dbias + 3u * n + 1u, (double)gv);
    atomicAdd(dbias + 3u * n + 2u, (double)gw);
}

// Vector-Jacobian product of one dual-time trilinear sample: given lambda of
// its (u, v, w), returns lambda . d(u, v, w)/d(x, y, z) and adds lambda x
// corner weight to the bias gradient of each corner node (the bias enters
// both frames, whose time weights sum to one).  Called by the whole warp;
// lanes with valid == false contribute nothing.  The bias terms of lanes
// whose samples share a corner set are summed across the warp first, and
// eight lanes then add one corner each to the CTA's table.
__device__ __forceinline__ float3 sample_vjp(const StepArgs& a, const Levels& lvl, bool valid, float x, float y,
                                             float z, float alpha, float lu, float lv, float lw,
                                             double* __restrict__ dbias, const BiasTable& table) {
    uint32_t x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    axis_bracket(x, a.nx, x0, x1, tx);
    axis_bracket(y, a.ny, y0, y1, ty);
    const float lev = meters_to_level(lvl, z);
    axis_bracket(lev, a.nz, z0, z1, tz);
    const float ix = (x > 0.0f && x < (float)(a.nx - 1u)) ? 1.0f : 0.0f;
    const float iy = (y > 0.0f && y < (float)(a.ny - 1u)) ? 1.0f : 0.0f;
    const float iz = (lev > 0.0f && lev < (float)(a.nz - 1u))
                         ? level_slope(lvl, z) : 0.0f;
    const uint32_t xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
    const float wx[2] = {1.0f - tx, tx}, wy[2] = {1.0f - ty, ty}, wz[2] = {1.0f - tz, tz};
    const float ta = 1.0f - alpha;
    // a lane whose lambda is zero (a particle that reaches no receptor after
    // this step) adds nothing: it loads no corners and joins no group
    const bool act = valid && (lu != 0.0f || lv != 0.0f || lw != 0.0f);
    float f[2][2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                float fv = 0.0f;
                if (act) {
                    const Node v = ld_node(a.bracket, (xs[i] * a.ny + ys[j]) * a.nz + zs[k]);
                    fv = lu * (ta * v.uv0.x + alpha * v.uv1.x) + lv * (ta * v.uv0.y + alpha * v.uv1.y) +
                         lw * (ta * v.w01.x + alpha * v.w01.y);
                }
                f[i][j][k] = fv;
            }
    if (dbias) {
        const uint32_t key = act ? (x0 * a.ny + y0) * a.nz + z0 : 0xffffffffu;
        const unsigned lane = threadIdx.x & 31u;
        unsigned pending = __ballot_sync(0xffffffffu, act);
        while (pending) {
            const int src = __ffs(pending) - 1;
            const uint32_t k0 = __shfl_sync(0xffffffffu, key, src);
            const bool mine = act && key == k0;
            const unsigned grp = __ballot_sync(0xffffffffu, mine);
            float v[24];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const float w = mine ? wx[c >> 2] * wy[(c >> 1) & 1] * wz[c & 1] : 0.0f;
                v[3 * c] = w * lu; v[3 * c + 1] = w * lv; v[3 * c + 2] = w * lw;
            }
            warp_sum24(v, lane);
            // the group's corner set is the source lane's; lane 4c issues corner c
            const uint32_t cx = __shfl_sync(0xffffffffu, x1, src), cy = __shfl_sync(0xffffffffu, y1, src);
            const uint32_t cz = __shfl_sync(0xffffffffu, z1, src);
            if ((lane & 3u) == 0u && (v[0] != 0.0f || v[1] != 0.0f || v[2] != 0.0f)) {
                const uint32_t c = lane >> 2;
                const uint32_t bx = k0 / (a.ny * a.nz), by = (k0 / a.nz) % a.ny, bz = k0 % a.nz;
                const uint32_t n = (((c >> 2) ? cx : bx) * a.ny + (((c >> 1) & 1u) ? cy : by)) * a.nz +
                                   ((c & 1u) ? cz : bz);
                bias_add(table, n, v[0], v[1], v[2], dbias);
            }
            pending &= ~grp;
        }
    }
    float gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k) gx += wy[j] * wz[k] * (f[1][j][k] - f[0][j][k]);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int k = 0; k < 2; ++k) gy += wx[i] * wz[k] * (f[i][1][k] - f[i][0][k]);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) gz += wx[i] * wy[j] * (f[i][j][1] - f[i][j][0]);
    return make_float3(gx * ix, gy * iy, gz * iz);
}

// dL/d(output state) of the receptor term of a sampling step.
__device__ __forceinline__ void receptor_seed(const Receptors& r, uint32_t inst, float x, float y, float z, float m,
                                              float& sx, float& sy, float& sz, float& sm) {
    sx = sy = sz = sm = 0.0f;
    const Cic c = cic(r, x, y, z);
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
            const int rr = receptor_at(r, inst, c.i0 + di, c.j0 + dj);
            if (rr < 0) continue;
            const float g = r.g[rr];
            const float wxy = c.wx[di] * c.wy[dj];
            sm += g * (wxy * c.v);
            sx += g * m * ((di ? 1.0f : -1.0f) * c.wy[dj] * c.v);
            sy += g * m * (c.wx[di] * (dj ? 1.0f : -1.0f) * c.v);
            sz += g * m * (wxy * c.dv);
        }
}

// The reverse of step `slice`'s tape.  One work item is 256 slots of one
// scenario, so a warp's lanes share the scenario: the release gradients are
// summed across the warp first.
__global__ void __launch_bounds__(256, 4) inverse_adjoint_kernel(StepArgs a, const BatchState* st,
                                                                 const ScenDev* __restrict__ sc,
                                                                 const uint2* __restrict__ items, uint32_t n_items,
                                                                 uint32_t* work, TapeBase tb, uint32_t slice,
                                                                 LamArrays lam, Receptors r,
                                                                 double* __restrict__ dbias,
                                                                 double* __restrict__ dsrc) {
    extern __shared__ float s_levels[];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_bias_key[kBiasTable];
    __shared__ float s_bias_g[3 * kBiasTable];
    const Levels lvl = stage_levels(a, s_levels);
    for (uint32_t i = threadIdx.x; i < kBiasTable; i += blockDim.x) {
        s_bias_key[i] = kBiasEmpty;
        s_bias_g[3u * i] = 0.0f;
        s_bias_g[3u * i + 1u] = 0.0f;
        s_bias_g[3u * i + 2u] = 0.0f;
    }
    const BiasTable table{s_bias_key, s_bias_g};
    const float alpha = st->alpha;
    const bool output = r.every != 0 && (st->step + 1u) % r.every == 0u;
    const float kx = a.xs * a.dt, ky = a.ys * a.dt, kz = a.zs * a.dt;
    TapeArrays tape;
#pragma unroll
    for (int f = 0; f < TAPE_FIELDS; ++f) tape.f[f] = tb.field(slice, f);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(work, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= n_items) break;
        const uint2 w = items[it];
        const ScenDev& d = sc[w.x];
        const uint32_t local = w.y + threadIdx.x;
        const uint32_t p = d.offset + local;
        const uint32_t fl = local < d.released ? reinterpret_cast<const uint32_t*>(tape.f[T_FLAGS])[p] : 0u;
        const bool valid = (fl & TAPE_ACTIVE) != 0u;
        if (__ballot_sync(0xffffffffu, valid) == 0u) continue;
        float lx = 0.0f, ly = 0.0f, lz = 0.0f, ltu = 0.0f, ltv = 0.0f, ltw = 0.0f, lm = 0.0f;
        float zz = 0.0f, ztw = 0.0f, wz = 0.0f, wtw = 0.0f, uz = 0.0f, uu = 0.0f, vz = 0.0f, vv = 0.0f;
        float px = 0.0f, py = 0.0f, pz = 0.0f, x0 = 0.0f, y0 = 0.0f, z0 = 0.0f;
        if (valid) {
            lx = lam.f[L_X][p]; ly = lam.f[L_Y][p]; lz = lam.f[L_Z][p];
            ltu = lam.f[L_TU][p]; ltv = lam.f[L_TV][p]; ltw = lam.f[L_TW][p];
            lm = lam.f[L_M][p];
            if (output) {
                // the receptor term of this step's output state
                float sx, sy, sz, sm;
                receptor_seed(r, d.instance, tape.f[T_X2][p], tape.f[T_Y2][p], tape.f[T_Z2][p], tape.f[T_M2][p],
                              sx, sy, sz, sm);
                lx += sx; ly += sy; lz += sz; lm += sm;
            }
            lm = lm * tape.f[T_SURV][p];
            zz = tape.f[T_ZZ][p]; ztw = tape.f[T_ZTW][p]; wz = tape.f[T_WZ][p]; wtw = tape.f[T_WTW][p];
            uz = tape.f[T_UZ][p]; uu = tape.f[T_UU][p]; vz = tape.f[T_VZ][p]; vv = tape.f[T_VV][p];
            px = tape.f[T_PX][p]; py = tape.f[T_PY][p]; pz = tape.f[T_PZ][p];
            x0 = tape.f[T_X0][p]; y0 = tape.f[T_Y0][p]; z0 = tape.f[T_Z0][p];
        }
        // turbulence: (z1, tu, tv, tw) -> (z2, tu', tv', tw')
        const float lz1 = lz * zz + ltw * wz + ltu * uz + ltv * vz;
        const float ltw0 = lz * ztw + ltw * wtw;
        float ltu0 = ltu * uu;
        float ltv0 = ltv * vv;
        // advection: x1 = clamp(x0 + cu kx), cu = (u0 + u1) / 2, u0 = s0.u + tu, u1 = s1.u + tu
        const float gx1 = (fl & ADV_X1) ? lx : 0.0f;
        const float gy1 = (fl & ADV_Y1) ? ly : 0.0f;
        const float gz1 = (fl & ADV_Z1) ? lz1 : 0.0f;
        float lx0 = gx1, ly0 = gy1, lz0 = gz1;
        float lu0 = 0.5f * gx1 * kx, lv0 = 0.5f * gy1 * ky, lw0 = 0.5f * gz1 * kz;
        const float lu1 = lu0, lv1 = lv0, lw1 = lw0;
        ltu0 += lu1;
        ltv0 += lv1;
        const float3 g1 = sample_vjp(a, lvl, valid, px, py, pz, alpha, lu1, lv1, lw1, dbias, table);
        const float gpx = (fl & ADV_PX) ? g1.x : 0.0f;
        const float gpy = (fl & ADV_PY) ? g1.y : 0.0f;
        const float gpz = (fl & ADV_PZ) ? g1.z : 0.0f;
        lx0 += gpx; lu0 += gpx * kx;
        ly0 += gpy; lv0 += gpy * ky;
        lz0 += gpz; lw0 += gpz * kz;
        ltu0 += lu0;
        ltv0 += lv0;
        const float3 g0 = sample_vjp(a, lvl, valid, x0, y0, z0, alpha, lu0, lv0, lw0, dbias, table);
        lx0 += g0.x; ly0 += g0.y; lz0 += g0.z;
        if (valid) {
            lam.f[L_X][p] = lx0; lam.f[L_Y][p] = ly0; lam.f[L_Z][p] = lz0;
            lam.f[L_TU][p] = ltu0; lam.f[L_TV][p] = ltv0; lam.f[L_TW][p] = ltw0;
            lam.f[L_M][p] = lm;
        }
        // released this step: the adjoint is the gradient of the release state
        const bool rel = valid && local >= d.rel_lo && local < d.rel_hi;
        if (__ballot_sync(0xffffffffu, rel)) {
            const float sx = warp_sum(rel ? lx0 : 0.0f), sy = warp_sum(rel ? ly0 : 0.0f);
            const float sz = warp_sum(rel ? lz0 : 0.0f), sm = warp_sum(rel ? lm : 0.0f);
            if ((threadIdx.x & 31u) == 0u) {
                double* g = dsrc + 4u * w.x;
                atomicAdd(g + 0, (double)sx);
                atomicAdd(g + 1, (double)sy);
                atomicAdd(g + 2, (double)sz);
                atomicAdd(g + 3, (double)sm);
            }
        }
    }
    // the loop ends for the whole CTA together: flush the bias table
    if (dbias) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kBiasTable; i += blockDim.x) {
            const uint32_t n = s_bias_key[i];
            if (n != kBiasEmpty) {
                atomicAdd(dbias + 3u * n + 0u, (double)s_bias_g[3u * i]);
                atomicAdd(dbias + 3u * n + 1u, (double)s_bias_g[3u * i + 1u]);
                atomicAdd(dbias + 3u * n + 2u, (double)s_bias_g[3u * i + 2u]);
            }
        }
    }
}

__global__ void __launch_bounds__(256) add_bias_kernel(const float4* __restrict__ raw, const float* __restrict__ bias,
                                                       uint32_t nodes, uint32_t frames, float4* __restrict__ out) {
    const size_t total = (size_t)nodes * frames;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t n = (uint32_t)(i % nodes);
        const float4 v = raw[i];
        out[i] = bias ? make_float4(v.x + bias[3u * n], v.y + bias[3u * n + 1u], v.z + bias[3u * n + 2u], v.w) : v;
    }
}

__global__ void __launch_bounds__(256) to_float_kernel(const double* __restrict__ in, size_t n, float* __restrict__ out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// Population fields a checkpoint keeps: everything the step and the release
// read.
constexpr int kCkptFields[] = {FPG_FIELD_POS_X, FPG_FIELD_POS_Y,  FPG_FIELD_POS_Z,  FPG_FIELD_CELL_X,
                               FPG_FIELD_CELL_Y, FPG_FIELD_FLAGS, FPG_FIELD_MASS0,  FPG_FIELD_TURB_U,
                               FPG_FIELD_TURB_V, FPG_FIELD_TURB_W, FPG_FIELD_CBT};
constexpr int kNumCkptFields = sizeof(kCkptFields) / sizeof(kCkptFields[0]);

struct InverseData {
    fpg_inverse_config cfg{};
    uint32_t n_instances = 1;
    std::vector<fpg_receptor> receptors;
    int32_t* rmap = nullptr;
    double* sim = nullptr;
    uint32_t* last_hit = nullptr;        // per slot, see Receptors
    float* g = nullptr;
    size_t nodes = 0;
    float4* ring_raw = nullptr;
    float* bias = nullptr;
    bool has_bias = false;
    bool tape_in_forward = false;        // checkpoint_every == 0
    uint32_t slices = 0;                 // tape slices: all steps, or K x max(W, 1)
    uint32_t window = 0;                 // K: steps per checkpoint window (all steps when taped)
    uint32_t n_windows = 0;              // windows of the run (1 when taped)
    uint32_t tail_windows = 0;           // W: last windows taped in the forward
    uint32_t n_ckpt = 0;
    uint32_t* ckpt = nullptr;            // n_ckpt * kNumCkptFields * capacity
    BatchState* ckpt_st = nullptr;
    ScenDev* ckpt_sc = nullptr;
    BatchState* st_all = nullptr;        // post-advance state per tape slice
    ScenDev* sc_all = nullptr;
    float* tape = nullptr;               // slices * TAPE_FIELDS * capacity
    float* lam = nullptr;                // LAM_FIELDS * capacity
    double* dbias = nullptr;
    float* dbias_f = nullptr;            // float copy for the host
    double* dsrc = nullptr;
    uint2* items = nullptr;              // 256-slot work items
    uint32_t n_items = 0;
    uint32_t* work_rev = nullptr;        // one work counter per tape slice for the reverse sweep
    // start time of the met bracket packed in device memory (INT64_MIN: unknown)
    int64_t packed_ta = INT64_MIN;
    bool forward_done = false;
    uint64_t bytes = 0;
    uint32_t grid_adj = 0;               // the reverse's persistent grid: SMs x resident CTAs
    // one taped step (pre, snapshot, tape pass, [sampling], end), captured
    cudaGraph_t tape_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t tape_exec[2] = {nullptr, nullptr};
    uint64_t tape_launches[2] = {0, 0};

    Receptors receptors_args(uint32_t nx, uint32_t ny) const {
        Receptors r;
        r.rmap = rmap;
        r.nx = nx; r.ny = ny; r.cells = nx * ny;
        r.ztop = cfg.receptor_top_m;
        r.ramp = cfg.receptor_ramp_m;
        r.every = cfg.sample_every_steps;
        r.g = g;
        r.sim = sim;
        r.last_hit = last_hit;
        return r;
    }
};

void enqueue_inverse_sample(fpg_batch* b, cudaStream_t s) {
    InverseData* inv = b->inv;
    const Receptors r = inv->receptors_args((uint32_t)b->met->nx, (uint32_t)b->met->ny);
    inverse_sample_kernel<<<b->ctx->sm_count * 8, 256, 0, s>>>(b->st, b->sc, inv->items, inv->n_items,
                                                              pop_fields(b), r);
    b->ctx->count(1);
}

}  // namespace fpg

using namespace fpg;

struct fpg_inverse {
    fpg_batch* b = nullptr;
    InverseData d;
};

static TapeBase tape_base(fpg_inverse* v) { return TapeBase{v->d.tape, v->b->capacity, v->d.slices}; }

static LamArrays lam_arrays(fpg_inverse* v) {
    LamArrays l;
    for (int f = 0; f < LAM_FIELDS; ++f) l.f[f] = v->d.lam + (size_t)f * v->b->capacity;
    return l;
}

// One taped step: the forward step with the tape pass in place of the plain
// particle pass; `sample` adds the receptor sampling (forward runs).
// The recompute (sample == false) steps only the slots whose adjoint is still
// non-zero (live).
static void enqueue_taped_step(fpg_inverse* v, bool sample, cudaStream_t s) {
    fpg_batch* b = v->b;
    InverseData& d = v->d;
    enqueue_pre(b, s);
    inverse_snapshot_kernel<<<1, 256, 0, s>>>(b->st, b->sc, (uint32_t)b->scen.size(), d.slices, d.st_all, d.sc_all);
    inverse_tape_kernel<<<std::max(d.n_items, 1u), 256, 0, s>>>(make_step_args(b), b->st, b->sc, d.items, d.n_items,
                                                                tape_base(v), d.cfg.sample_every_steps,
                                                                sample ? nullptr : d.last_hit);
    b->ctx->count(2);
    if (sample) enqueue_inverse_sample(b, s);
    enqueue_end(b, s);
}

static fpg_status ensure_tape_graph(fpg_inverse* v, int sample) {
    InverseData& d = v->d;
    if (d.tape_exec[sample]) return FPG_OK;
    cudaStream_t s = v->b->ctx->stream;
    FPG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = v->b->ctx->launches.load();
    enqueue_taped_step(v, sample != 0, s);
    d.tape_launches[sample] = v->b->ctx->launches.load() - before;
    v->b->ctx->launches.fetch_sub(d.tape_launches[sample]);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) return cuda_status(e);
    d.tape_graph[sample] = g;
    FPG_CUDA(cudaGraphInstantiate(&d.tape_exec[sample], g, 0));
    return FPG_OK;
}

static fpg_status rebuild_ring(fpg_inverse* v) {
    const uint32_t frames = v->b->cfg.n_frames;
    add_bias_kernel<<<v->b->ctx->sm_count * 4, 256, 0, v->b->ctx->stream>>>(
        v->d.ring_raw, v->d.has_bias ? v->d.bias : nullptr, (uint32_t)v->d.nodes, frames, v->b->ring);
    v->b->ctx->count(1);
    FPG_CHECK_LAUNCH();
    v->d.forward_done = false;
    v->d.packed_ta = INT64_MIN;             // the ring changed under the packed bracket
    return FPG_OK;
}

static cudaError_t save_checkpoint(fpg_inverse* v, uint32_t c) {
    fpg_batch* b = v->b;
    cudaStream_t s = b->ctx->stream;
    const size_t cap = b->capacity;
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < kNumCkptFields && e == cudaSuccess; ++f)
        e = cudaMemcpyAsync(v->d.ckpt + ((size_t)c * kNumCkptFields + f) * cap, b->pop->field[kCkptFields[f]],
                            cap * 4, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v->d.ckpt_st + c, b->st, sizeof(BatchState), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(v->d.ckpt_sc + (size_t)c * b->scen.size(), b->sc, b->scen.size() * sizeof(ScenDev),
                            cudaMemcpyDeviceToDevice, s);
    return e;
}

static cudaError_t restore_checkpoint(fpg_inverse* v, uint32_t c) {
    fpg_batch* b = v->b;
    cudaStream_t s = b->ctx->stream;
    const size_t cap = b->capacity;
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < kNumCkptFields && e == cudaSuccess; ++f)
        e = cudaMemcpyAsync(b->pop->field[kCkptFields[f]], v->d.ckpt + ((size_t)c * kNumCkptFields + f) * cap,
                            cap * 4, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->st, v->d.ckpt_st + c, sizeof(BatchState), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->sc, v->d.ckpt_sc + (size_t)c * b->scen.size(), b->scen.size() * sizeof(ScenDev),
                            cudaMemcpyDeviceToDevice, s);
    // the device bracket and wet fields hold whatever was packed last: make
    // the next step repack them
    if (e == cudaSuccess)
        e = cudaMemsetAsync(reinterpret_cast<char*>(b->st) + offsetof(BatchState, have_bracket), 0, sizeof(int32_t), s);
    return e;
}

extern "C" fpg_status fpg_inverse_destroy(fpg_inverse* v) {
    if (!v) return FPG_OK;
    if (v->b) {
        cudaStreamSynchronize(v->b->ctx->stream);
        v->b->inv = nullptr;
    }
    InverseData& d = v->d;
    for (int k = 0; k < 2; ++k) {
        if (d.tape_exec[k]) cudaGraphExecDestroy(d.tape_exec[k]);
        if (d.tape_graph[k]) cudaGraphDestroy(d.tape_graph[k]);
    }
    cudaFree(d.rmap); cudaFree(d.sim); cudaFree(d.last_hit); cudaFree(d.g); cudaFree(d.ring_raw); cudaFree(d.bias);
    cudaFree(d.ckpt); cudaFree(d.ckpt_st); cudaFree(d.ckpt_sc); cudaFree(d.st_all); cudaFree(d.sc_all);
    cudaFree(d.tape); cudaFree(d.lam); cudaFree(d.dbias); cudaFree(d.dbias_f); cudaFree(d.dsrc);
    cudaFree(d.items); cudaFree(d.work_rev);
    fpg_batch_destroy(v->b);
    delete v;
    return FPG_OK;
}

extern "C" fpg_status fpg_inverse_create(fpg_ctx* ctx, const fpg_inverse_config* cfg, const fpg_batch_scenario* src,
                                         const uint32_t* src_instance, size_t n_src, size_t nx, size_t ny, size_t nz,
                                         const float* heights, const fpg_receptor* rec, size_t n_rec,
                                         fpg_inverse** out) {
    if (!ctx || !cfg || !src || !out || n_src == 0 || (n_rec && !rec)) return FPG_ERR_INVALID_ARGUMENT;
    if (!(cfg->receptor_ramp_m > 0.0f) || !std::isfinite(cfg->receptor_top_m)) return FPG_ERR_INVALID_ARGUMENT;
    uint32_t n_inst = 1;
    if (src_instance)
        for (size_t s = 0; s < n_src; ++s) n_inst = std::max(n_inst, src_instance[s] + 1u);
    for (size_t r = 0; r < n_rec; ++r)
        if (rec[r].instance >= n_inst || rec[r].i >= nx || rec[r].j >= ny) return FPG_ERR_INVALID_ARGUMENT;
    fpg_batch_config bc = cfg->batch;
    bc.out_nx = bc.out_ny = bc.out_nz = 0;
    bc.outheights = nullptr;
    bc.output_every_steps = 0;
    fpg_inverse* v = new fpg_inverse();
    fpg_status st = fpg_batch_create(ctx, &bc, src, n_src, nx, ny, nz, heights, &v->b);
    if (st != FPG_OK) { delete v; return st; }
    fpg_batch* b = v->b;
    InverseData& d = v->d;
    d.cfg = *cfg;
    d.n_instances = n_inst;
    d.receptors.assign(rec, rec + n_rec);
    for (size_t s = 0; s < n_src; ++s) b->scen[s].instance = src_instance ? src_instance[s] : 0u;
    d.nodes = nx * ny * nz;
    const size_t cells = nx * ny, cap = b->capacity;
    d.tape_in_forward = cfg->checkpoint_every == 0;
    const uint32_t K = std::max<uint32_t>(1u, d.tape_in_forward
                                                  ? (uint32_t)b->total_steps
                                                  : (uint32_t)std::min<uint64_t>(cfg->checkpoint_every,
                                                                                 b->total_steps));
    d.window = K;
    d.n_windows = d.tape_in_forward ? 1u : (uint32_t)((b->total_steps + K - 1) / K);
    d.tail_windows = d.tape_in_forward ? 1u : std::min<uint32_t>(cfg->tape_tail_windows, d.n_windows);
    // tail windows are taped in the forward, earlier ones recomputed into
    // the same slices (step % slices) after the tail has been reversed
    d.slices = d.tape_in_forward ? K : K * std::max<uint32_t>(d.tail_windows, 1u);
    d.n_ckpt = d.tape_in_forward ? 0u : d.n_windows - d.tail_windows;
    // work items of 256 slots for the tape and adjoint kernels
    std::vector<uint2> items;
    for (size_t s = 0; s < n_src; ++s)
        for (uint32_t l = 0; l < b->scen[s].capacity; l += TILE) items.push_back(make_uint2((uint32_t)s, l));
    d.n_items = (uint32_t)items.size();
    std::vector<int32_t> rmap((size_t)n_inst * cells, -1);
    for (size_t r = 0; r < n_rec; ++r) rmap[(size_t)rec[r].instance * cells + rec[r].i * ny + rec[r].j] = (int32_t)r;
    auto alloc = [&](void** p, size_t bytes) {
        d.bytes += bytes;
        return cudaMalloc(p, bytes ? bytes : 4);
    };
    cudaError_t e = alloc((void**)&d.rmap, rmap.size() * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.sim, std::max<size_t>(n_rec, 1) * 8);
    if (e == cudaSuccess) e = alloc((void**)&d.last_hit, cap * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.g, std::max<size_t>(n_rec, 1) * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.ring_raw, d.nodes * bc.n_frames * sizeof(float4));
    if (e == cudaSuccess) e = alloc((void**)&d.bias, d.nodes * 3 * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.ckpt, (size_t)d.n_ckpt * kNumCkptFields * cap * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.ckpt_st, std::max<uint32_t>(d.n_ckpt, 1) * sizeof(BatchState));
    if (e == cudaSuccess) e = alloc((void**)&d.ckpt_sc, (size_t)std::max<uint32_t>(d.n_ckpt, 1) * n_src * sizeof(ScenDev));
    const uint32_t S = d.slices;
    if (e == cudaSuccess) e = alloc((void**)&d.st_all, S * sizeof(BatchState));
    if (e == cudaSuccess) e = alloc((void**)&d.sc_all, (size_t)S * n_src * sizeof(ScenDev));
    if (e == cudaSuccess) e = alloc((void**)&d.tape, (size_t)S * TAPE_FIELDS * cap * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.lam, (size_t)LAM_FIELDS * cap * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.dbias, d.nodes * 3 * 8);
    if (e == cudaSuccess) e = alloc((void**)&d.dbias_f, d.nodes * 3 * 4);
    if (e == cudaSuccess) e = alloc((void**)&d.dsrc, n_src * 4 * 8);
    if (e == cudaSuccess) e = alloc((void**)&d.items, items.size() * sizeof(uint2));
    if (e == cudaSuccess) e = alloc((void**)&d.work_rev, (size_t)S * 4);
    cudaStream_t s = ctx->stream;
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.rmap, rmap.data(), rmap.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d.items, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.bias, 0, d.nodes * 3 * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d.ring_raw, 0, d.nodes * bc.n_frames * sizeof(float4), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    int per_sm_adj = 0;
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_adj, inverse_adjoint_kernel, 256,
                                                          nz * sizeof(float) + FPG_LEVEL_BUCKETS);
    if (e != cudaSuccess) {
        fpg_inverse_destroy(v);
        return cuda_status(e);
    }
    d.grid_adj = (uint32_t)ctx->sm_count * (uint32_t)std::max(per_sm_adj, 1);
    b->inv = &d;
    *out = v;
    return FPG_OK;
}

extern "C" fpg_status fpg_inverse_upload_frame(fpg_inverse* v, uint32_t k, const float* u, const float* vv,
                                               const float* w, const fpg_surface_cell* surface, const float* precip) {
    if (!v) return FPG_ERR_INVALID_ARGUMENT;
    fpg_status st = fpg_batch_upload_frame(v->b, k, u, vv, w, surface, precip);
    if (st != FPG_OK) return st;
    FPG_CUDA(cudaMemcpyAsync(v->d.ring_raw + (size_t)k * v->d.nodes, v->b->ring + (size_t)k * v->d.nodes,
                             v->d.nodes * sizeof(float4), cudaMemcpyDeviceToDevice, v->b->ctx->stream));
    return rebuild_ring(v);
}

extern "C" fpg_status fpg_inverse_set_wind_bias(fpg_inverse* v, const float* bias) {
    if (!v) return FPG_ERR_INVALID_ARGUMENT;
    v->d.has_bias = bias != nullptr;
    if (bias)
        FPG_CUDA(cudaMemcpyAsync(v->d.bias, bias, v->d.nodes * 3 * 4, cudaMemcpyHostToDevice, v->b->ctx->stream));
    return rebuild_ring(v);
}

extern "C" fpg_status fpg_inverse_set_sources(fpg_inverse* v, const double* mass, const double* pos) {
    if (!v) return FPG_ERR_INVALID_ARGUMENT;
    fpg_batch* b = v->b;
    std::vector<ScenDev> next = b->scen;
    for (size_t s = 0; s < next.size(); ++s) {
        ScenDev& d = next[s];
        if (mass) {
            if (!std::isfinite(mass[s])) return FPG_ERR_INVALID_ARGUMENT;
            d.mass_per_particle = (float)(mass[s] / (double)d.count);
        }
        if (pos) {
            const double dlon = pos[3 * s] - d.lon_min, dlat = pos[3 * s + 1] - d.lat_min, dz = pos[3 * s + 2] - d.z_min;
            d.lon_min += dlon; d.lon_max += dlon;
            d.lat_min += dlat; d.lat_max += dlat;
            d.z_min += dz; d.z_max += dz;
            if (check_release_grid(d, b->cfg.release_grid) != FPG_OK) return FPG_ERR_OUT_OF_GRID;
        }
    }
    b->scen = next;
    v->d.forward_done = false;
    return FPG_OK;
}

// Start of the met bracket that step k runs in: batch_advance_kernel's
// formula at t = start + k dt (at a frame time the bracket ending there).
static int64_t step_bracket_start(const fpg_batch* b, uint64_t k) {
    const int64_t start = b->cfg.start_seconds, fs = b->cfg.frame_seconds;
    const int64_t t = start + (int64_t)k * b->cfg.timestep_seconds;
    int64_t i = (t - start) / fs;
    if (t - start == i * fs && i > 0) i -= 1;
    return start + i * fs;
}

extern "C" fpg_status fpg_inverse_forward(fpg_inverse* v, double* simulated) {
    if (!v) return FPG_ERR_INVALID_ARGUMENT;
    fpg_batch* b = v->b;
    InverseData& d = v->d;
    cudaStream_t s = b->ctx->stream;
    fpg_status st = batch_reset(b);
    if (st != FPG_OK) return st;
    FPG_CUDA(cudaMemsetAsync(d.sim, 0, std::max<size_t>(d.receptors.size(), 1) * 8, s));
    FPG_CUDA(cudaMemsetAsync(d.last_hit, 0, v->b->capacity * 4, s));
    if (d.tape_in_forward) {
        if ((st = ensure_tape_graph(v, 1)) != FPG_OK) return st;
        for (uint64_t k = 0; k < b->total_steps; ++k) {
            FPG_CUDA(cudaGraphLaunch(d.tape_exec[1], s));
            b->ctx->count(d.tape_launches[1]);
        }
    } else {
        if ((st = ensure_graph(b)) != FPG_OK) return st;
        if (d.tail_windows && (st = ensure_tape_graph(v, 1)) != FPG_OK) return st;
        const uint32_t K = d.window;
        const uint64_t k_tail = (uint64_t)(d.n_windows - d.tail_windows) * K;
        for (uint64_t k = 0; k < b->total_steps; ++k) {
            if (k < k_tail) {
                if (k % K == 0) FPG_CUDA(save_checkpoint(v, (uint32_t)(k / K)));
                FPG_CUDA(cudaGraphLaunch(b->exec, s));
                b->ctx->count(b->graph_launches);
            } else {                         // a tail window: record its tape now
                FPG_CUDA(cudaGraphLaunch(d.tape_exec[1], s));
                b->ctx->count(d.tape_launches[1]);
            }
        }
    }
    b->steps_done = b->total_steps;
    // the step kernels left the bracket of the last step packed
    if (b->total_steps) d.packed_ta = step_bracket_start(b, b->total_steps - 1);
    if (simulated && !d.receptors.empty())
        FPG_CUDA(cudaMemcpyAsync(simulated, d.sim, d.receptors.size() * 8, cudaMemcpyDeviceToHost, s));
    FPG_CUDA(cudaStreamSynchronize(s));
    int32_t err = 0;
    fpg_batch_errors(b, &err);
    if (err) return FPG_ERR_OUT_OF_GRID;
    d.forward_done = true;
    return FPG_OK;
}

extern "C" fpg_status fpg_inverse_backward(fpg_inverse* v, const double* d_sim, double* d_mass, double* d_pos,
                                           float* d_bias) {
    if (!v || (!d_sim && !v->d.receptors.empty())) return FPG_ERR_INVALID_ARGUMENT;
    InverseData& d = v->d;
    if (!d.forward_done) return FPG_ERR_NOT_READY;
    fpg_batch* b = v->b;
    cudaStream_t s = b->ctx->stream;
    const size_t n_src = b->scen.size(), cap = b->capacity;
    std::vector<float> g(std::max<size_t>(d.receptors.size(), 1), 0.0f);
    for (size_t r = 0; r < d.receptors.size(); ++r) g[r] = (float)d_sim[r];
    FPG_CUDA(cudaMemcpyAsync(d.g, g.data(), g.size() * 4, cudaMemcpyHostToDevice, s));
    FPG_CUDA(cudaMemsetAsync(d.lam, 0, (size_t)LAM_FIELDS * cap * 4, s));
    FPG_CUDA(cudaMemsetAsync(d.dbias, 0, d.nodes * 3 * 8, s));
    FPG_CUDA(cudaMemsetAsync(d.dsrc, 0, n_src * 4 * 8, s));
    const StepArgs a = make_step_args(b);
    const Receptors rargs = d.receptors_args((uint32_t)b->met->nx, (uint32_t)b->met->ny);
    const LamArrays lam = lam_arrays(v);
    const TapeBase tb = tape_base(v);
    const size_t smem = level_smem_bytes(b->met);
    const uint64_t n = b->total_steps;
    const uint32_t K = d.window, S = d.slices;
    const int64_t windows = d.n_windows;
    // windows below this one are recomputed from their checkpoints
    const int64_t first_taped = d.tape_in_forward ? 0 : (int64_t)(d.n_windows - d.tail_windows);
    fpg_status st = FPG_OK;
    if (first_taped > 0 && (st = ensure_tape_graph(v, 0)) != FPG_OK) return st;
    for (int64_t w = windows - 1; w >= 0; --w) {
        const uint64_t k0 = (uint64_t)w * K, k1 = std::min<uint64_t>(k0 + K, n);
        if (w < first_taped) {
            // taped recompute of the window from its checkpoint; it leaves the
            // bracket of its last step packed
            FPG_CUDA(restore_checkpoint(v, (uint32_t)w));
            for (uint64_t k = k0; k < k1; ++k) {
                FPG_CUDA(cudaGraphLaunch(d.tape_exec[0], s));
                b->ctx->count(d.tape_launches[0]);
            }
            d.packed_ta = step_bracket_start(b, k1 - 1);
        }
        // one work counter per slice, cleared once per window
        FPG_CUDA(cudaMemsetAsync(d.work_rev, 0, (size_t)S * 4, s));
        // reverse of the window; the bracket is repacked only where it changes
        for (uint64_t k = k1; k-- > k0;) {
            const uint32_t j = (uint32_t)(k % S);
            const int64_t ta = step_bracket_start(b, k);
            if (ta != d.packed_ta) {
                enqueue_pack_forced(b, d.st_all + j, s);
                d.packed_ta = ta;
            }
            inverse_adjoint_kernel<<<d.grid_adj, 256, smem, s>>>(a, d.st_all + j, d.sc_all + (size_t)j * n_src,
                                                                 d.items, d.n_items, d.work_rev + j, tb, j, lam,
                                                                 rargs, d_bias ? d.dbias : nullptr, d.dsrc);
            b->ctx->count(1);
            FPG_CHECK_LAUNCH();
        }
    }
    std::vector<double> src(n_src * 4);
    FPG_CUDA(cudaMemcpyAsync(src.data(), d.dsrc, n_src * 4 * 8, cudaMemcpyDeviceToHost, s));
    if (d_bias) {
        to_float_kernel<<<b->ctx->sm_count * 4, 256, 0, s>>>(d.dbias, d.nodes * 3, d.dbias_f);
        b->ctx->count(1);
        FPG_CUDA(cudaMemcpyAsync(d_bias, d.dbias_f, d.nodes * 3 * 4, cudaMemcpyDeviceToHost, s));
    }
    FPG_CUDA(cudaStreamSynchronize(s));
    const fpg_grid_domain& gd = b->cfg.release_grid;
    for (size_t k = 0; k < n_src; ++k) {
        if (d_mass) d_mass[k] = src[4 * k + 3] / (double)b->scen[k].count;
        if (d_pos) {
            d_pos[3 * k] = src[4 * k] / gd.dx;
            d_pos[3 * k + 1] = src[4 * k + 1] / gd.dy;
            d_pos[3 * k + 2] = src[4 * k + 2];
        }
    }
    // after a recompute the population holds the first window's recompute
    // and the tail slices are overwritten; a tape recorded entirely in the
    // forward stays valid for another backward
    if (first_taped > 0) d.forward_done = false;
    return FPG_OK;
}

extern "C" fpg_batch* fpg_inverse_batch(fpg_inverse* v) { return v ? v->b : nullptr; }

extern "C" uint64_t fpg_inverse_device_bytes(const fpg_inverse* v) { return v ? v->d.bytes : 0; }
