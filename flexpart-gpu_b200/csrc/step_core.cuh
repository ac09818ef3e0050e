// step_core.cuh -- the per-particle body of the fused step, shared by the
// single-population kernel (step.cu) and the batched scenario kernel
// (batch.cu).  See step.cu for the reference passes it replaces.
#pragma once

#include "fpg_internal.h"
#include "physics.cuh"
#include "dual.cuh"

namespace fpg {

struct StepArgs {
    int32_t* cell_x; int32_t* cell_y;
    float* pos_x; float* pos_y; float* pos_z;
    const uint32_t* flags;
    float* mass[4];
    float* vel_u; float* vel_v; float* vel_w;
    float* turb_u; float* turb_v; float* turb_w;
    int32_t* cbt;
    uint32_t n;
    int n_species;
    uint32_t stages;
    // advection
    const float4* bracket;
    const float* heights;
    const uint8_t* level_table;          // FPG_LEVEL_BUCKETS bytes when level_mode == LEVELS_TABLE
    float level_inv_w;
    uint32_t nx, ny, nz;
    int has_heights, level_mode;
    float alpha, dt, xs, ys, zs;
    // turbulence: the per-cell Hanna constants (pbl_cell)
    const CellHanna* hcell;
    uint32_t pnx, pny;
    float tdt, rho, zmin;
    uint32_t n_sub;
    uint32_t key0, key1;
    u32x4 counter;
    // deposition
    float href;
    int dry_mode;
    float dry_v;
    const float* dry_v_arr;
    float* dry_prob;
    int wet_mode;
    float wet_l, wet_f;
    const float* wet_l_arr;
    const float* wet_f_arr;
    const float2* wet_cells;
    uint32_t wnx, wny;
    float* wet_prob;
};

// How the level search runs: the reference's linear scan (heights not
// sorted), a binary search (sorted), or a bucket table plus a short scan
// (sorted with h[nz-1] > h[0]).  All three return the scan's index.
enum { LEVELS_SCAN = 0, LEVELS_BISECT = 1, LEVELS_TABLE = 2 };

// The search a met's heights allow (host side).
inline int level_mode(const fpg_met* m) {
    return m->level_table ? LEVELS_TABLE : m->monotonic ? LEVELS_BISECT : LEVELS_SCAN;
}

// The level heights and the bucket table where a kernel reads them: in
// global memory through L1 (global_levels), or staged in shared memory
// (stage_levels).
struct Levels {
    const float* h;
    const uint8_t* tab;
    float inv_w;
    uint32_t nz;
    int has, mode;
};

// The met's own arrays (a kernel with one particle per thread: every CTA
// would otherwise stage them for its 256 particles and wait at a barrier).
__device__ __forceinline__ Levels global_levels(const StepArgs& a) {
    return Levels{a.heights, a.level_table, a.level_inv_w, a.nz, a.has_heights, a.level_mode};
}

// Copies the level heights (and the bucket table) into shared memory at
// `smem` (level_smem_bytes of the met); the caller synchronises the block.
__device__ __forceinline__ Levels stage_levels(const StepArgs& a, float* smem) {
    for (uint32_t i = threadIdx.x; i < a.nz; i += blockDim.x) smem[i] = a.heights[i];
    uint32_t* tab = reinterpret_cast<uint32_t*>(smem + a.nz);
    if (a.level_mode == LEVELS_TABLE)
        for (uint32_t i = threadIdx.x; i < FPG_LEVEL_BUCKETS / 4u; i += blockDim.x)
            tab[i] = __ldg(reinterpret_cast<const uint32_t*>(a.level_table) + i);
    return Levels{smem, reinterpret_cast<const uint8_t*>(tab), a.level_inv_w, a.nz, a.has_heights, a.level_mode};
}

// The first k in [1, nz) with z <= h[k], nz if none (the loop of
// advection_dual_wind.wgsl:101-110), for z > h[0].
__device__ __forceinline__ uint32_t level_index(const Levels& L, float z) {
    const float* h = L.h;
    const uint32_t nz = L.nz;
    uint32_t k;
    if (L.mode == LEVELS_TABLE) {
        // every level below the table's entry lies under z (the entry is
        // taken one bucket low), so scanning up from it finds the same k
        const uint32_t b = min(__float2uint_rz((z - h[0]) * L.inv_w), FPG_LEVEL_BUCKETS - 1u);
        k = (uint32_t)L.tab[b] + 1u;
        while (k < nz && !(z <= h[k])) ++k;
    } else if (L.mode == LEVELS_BISECT) {
        uint32_t lo = 1u, hi = nz;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (z <= h[mid]) hi = mid; else lo = mid + 1u;
        }
        k = lo;
    } else {
        k = nz;
        for (uint32_t i = 1u; i < nz; ++i) if (z <= h[i]) { k = i; break; }
    }
    return k;
}

// meters_to_grid_level (advection_dual_wind.wgsl:94-117).
__device__ __forceinline__ float meters_to_level(const Levels& L, float z) {
    if (!L.has) return z;
    const float* h = L.h;
    const uint32_t nz = L.nz;
    const float h0 = h[0];
    if (z <= h0) return h0 > 0.0f ? sdiv(z, h0) : 0.0f;
    const uint32_t k = level_index(L, z);
    if (k >= nz) return (float)(nz - 1u);
    const float hprev = h[k - 1u];
    const float denom = h[k] - hprev;
    if (denom > 0.0f) return (float)(k - 1u) + sdiv(z - hprev, denom);
    return (float)(k - 1u);
}

// clamp_axis (advection_dual_wind.wgsl:130-138).
__device__ __forceinline__ void axis_bracket(float coord, uint32_t n, uint32_t& lo, uint32_t& hi, float& t) {
    const float c = clampf(coord, 0.0f, (float)(n - 1u));
    const float lf = floorf(c);
    lo = (uint32_t)lf;
    hi = min(lo + 1u, n - 1u);
    t = c - lf;
}

// sample_dual_{u,v,w} (advection_dual_wind.wgsl:142-236): trilinear in each
// frame, then lerp by alpha.  The x-lerps of one (y, z) corner pair are taken
// as soon as its two nodes arrive, which keeps the live registers at 16
// floats instead of 64 while giving the same roundings in the same order as
// the reference expression.  The six channels (u, v, w of both frames) are
// interpolated two at a time with the packed FP32 instructions of sm_100
// (__fmul2_rn / __ffma2_rn: each lane is one IEEE round-to-nearest multiply
// or fused multiply-add, so a lane's result is lerpf's bit for bit), on the
// register pairs the node load fills: (u0, v0), (u1, v1), (w0, w1).

// One bracket node is 32 bytes at a 32-byte aligned offset (cudaMalloc base,
// node stride 32 B), laid out (u0, v0, u1, v1, w0, w1, 0, 0) with frame 0
// the bracket's t0: one 256-bit load, whose last two lanes are not used.
struct Node { float2 uv0, uv1, w01; };

__device__ __forceinline__ Node ld_node(const float4* br, uint32_t n) {
    Node v;
    asm("{\n.reg .f32 pad<2>;\nld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,pad0,pad1}, [%6];\n}"
        : "=f"(v.uv0.x), "=f"(v.uv0.y), "=f"(v.uv1.x), "=f"(v.uv1.y), "=f"(v.w01.x), "=f"(v.w01.y)
        : "l"(br + 2u * n));
    return v;
}

// The node layout from two frames' (u, v, w, 0).
__device__ __forceinline__ void st_node(float4* br, uint32_t n, float4 f0, float4 f1) {
    br[2u * n] = make_float4(f0.x, f0.y, f1.x, f1.y);
    br[2u * n + 1u] = make_float4(f0.z, f1.z, 0.0f, 0.0f);
}

// lerpf on two lanes: fmaf(a, 1 - t, b * t) with s = (1 - t, 1 - t).
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 s, float2 t) {
    return __ffma2_rn(a, s, __fmul2_rn(b, t));
}

__device__ __forceinline__ Node lerp_node(const Node& a, const Node& b, float2 s, float2 t) {
    return Node{lerp2(a.uv0, b.uv0, s, t), lerp2(a.uv1, b.uv1, s, t), lerp2(a.w01, b.w01, s, t)};
}

__device__ __forceinline__ Node xpair(const float4* br, uint32_t na, uint32_t nb, float2 s, float2 t) {
    return lerp_node(ld_node(br, na), ld_node(br, nb), s, t);
}

__device__ __forceinline__ float3 sample_dual(const StepArgs& a, const Levels& lv, float x, float y, float z,
                                              float alpha) {
    uint32_t x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    axis_bracket(x, a.nx, x0, x1, tx);
    axis_bracket(y, a.ny, y0, y1, ty);
    axis_bracket(meters_to_level(lv, z), a.nz, z0, z1, tz);
    const uint32_t c00 = (x0 * a.ny + y0) * a.nz, c10 = (x1 * a.ny + y0) * a.nz;
    const uint32_t c01 = (x0 * a.ny + y1) * a.nz, c11 = (x1 * a.ny + y1) * a.nz;
    const float4* br = a.bracket;
    const float2 tx2 = make_float2(tx, tx), sx2 = make_float2(1.0f - tx, 1.0f - tx);
    const float2 ty2 = make_float2(ty, ty), sy2 = make_float2(1.0f - ty, 1.0f - ty);
    const float2 tz2 = make_float2(tz, tz), sz2 = make_float2(1.0f - tz, 1.0f - tz);
    // lerp(lerp(lerp(c000,c100,tx), lerp(c010,c110,tx), ty), lerp(lerp(c001,c101,tx), lerp(c011,c111,tx), ty), tz)
    const Node l00 = xpair(br, c00 + z0, c10 + z0, sx2, tx2);
    const Node l10 = xpair(br, c01 + z0, c11 + z0, sx2, tx2);
    const Node l0 = lerp_node(l00, l10, sy2, ty2);
    const Node l01 = xpair(br, c00 + z1, c10 + z1, sx2, tx2);
    const Node l11 = xpair(br, c01 + z1, c11 + z1, sx2, tx2);
    const Node l1 = lerp_node(l01, l11, sy2, ty2);
    const Node t = lerp_node(l0, l1, sz2, tz2);
    const float2 ta = make_float2(alpha, alpha), sa = make_float2(1.0f - alpha, 1.0f - alpha);
    const float2 uv = lerp2(t.uv0, t.uv1, sa, ta);
    return make_float3(uv.x, uv.y, lerpf(t.w01.x, t.w01.y, alpha));
}

// split_horizontal_coord (advection_dual_wind.wgsl:238-248).
__device__ __forceinline__ void split_coord(float coord, uint32_t n, int32_t& cell, float& frac) {
    const float c = clampf(coord, 0.0f, (float)(n - 1u));
    uint32_t ci = (uint32_t)floorf(c);
    float f = c - (float)ci;
    if (ci >= n - 1u) { ci = n - 1u; f = 0.0f; }
    cell = (int32_t)ci;
    frac = f;
}

// The Langevin updates as the fused shader applies them to Hanna outputs
// (sigma >= 0.01 and T_L >= 10 s by construction).
struct HannaLangevin {
    template <class T>
    __device__ static __forceinline__ T h(T prev, T sigma, T tl, float dt, float eta) {
        return langevin_h_t<T>(prev, sigma, tl, dt, eta);
    }
    template <class T>
    __device__ static __forceinline__ T v(T prev, T sigma_w, T tlw, T dsigwdz, float dt, float rho, float eta) {
        return langevin_v_t<T>(prev, sigma_w, tlw, dsigwdz, dt, rho, eta);
    }
};

// The same updates on caller-supplied HannaParams records (langevin.wgsl:
// 189-238, physics/langevin.rs:116-121,146-150): sigma and T_L pass through
// sanitize_positive and a zero T_L gives zero turbulence.  Float only.
struct RecordLangevin {
    __device__ static __forceinline__ float h(float prev, float sigma, float tl, float dt, float eta) {
        const float s = sanitize_positive(sigma), t = sanitize_positive(tl);
        return t == 0.0f ? 0.0f : langevin_h_t<float>(prev, s, t, dt, eta);
    }
    __device__ static __forceinline__ float v(float prev, float sigma_w, float tlw, float dsigwdz, float dt,
                                              float rho, float eta) {
        const float s = sanitize_positive(sigma_w), t = sanitize_positive(tlw);
        return t == 0.0f ? 0.0f : langevin_v_t<float>(prev, s, t, dsigwdz, dt, rho, eta);
    }
};

// Turbulence of one particle from its Hanna parameters
// (langevin_fused.wgsl:446-515, langevin.wgsl:350-421): horizontal Langevin
// updates, then the vertical sub-steps with ground and PBL-top reflection and
// the vertical Hanna re-evaluation between sub-steps.  A template over the
// scalar type (float for the step, the dual number of the adjoint for its
// Jacobian: same values, bit for bit), the update policy and the argument
// block (any type with tdt, rho, zmin and n_sub).
template <class T, class L, class A>
__device__ __forceinline__ void turbulence_from_hanna(const A& a, const CellHanna& cell, const HannaT<T>& hn,
                                                      float2 e_uv, float2 e_w01, float2 e_w23, T& pz, T& tu, T& tv,
                                                      T& tw, int32_t& cbt) {
    tu = L::h(tu, hn.sigu, hn.tlu, a.tdt, e_uv.x);
    tv = L::h(tv, hn.sigv, hn.tlv, a.tdt, e_uv.y);
    if (a.n_sub == 0u) {
        tw = L::v(tw, hn.sigw, hn.tlw, hn.dsigwdz, a.tdt, a.rho, e_w01.x);
        return;
    }
    const float dt_sub = sdiv(a.tdt, (float)a.n_sub);
    const float h = hn.h;
    const float zmin = a.zmin;
    T sigw = hn.sigw, dsigwdz = hn.dsigwdz, tlw = hn.tlw;
    for (uint32_t sub = 0; sub < a.n_sub; ++sub) {
        const float eta = sub == 0u ? e_w01.x : sub == 1u ? e_w01.y : sub == 2u ? e_w23.x : e_w23.y;
        tw = L::v(tw, sigw, tlw, dsigwdz, dt_sub, a.rho, eta);
        pz = pz + tw * dt_sub;
        if (h > zmin) {
            // the first bounce by selects (most sub-steps need none or one, and
            // a warp's lanes disagree on which), the loop only for the rest
            T z = pz;
            const bool lo = val(z) < zmin, hi = !lo && val(z) > h;
            const bool any = lo || hi;
            const T zr = lo ? T(2.0f * zmin - z) : T(2.0f * h - z);
            z = any ? zr : z;
            cbt = any ? -cbt : cbt;
            tw = any ? T(-tw) : tw;
            if (any && (val(z) < zmin || val(z) > h)) {
                for (int bounce = 1; bounce < 10; ++bounce) {
                    if (val(z) < zmin) { z = 2.0f * zmin - z; cbt = -cbt; tw = -tw; }
                    else if (val(z) > h) { z = 2.0f * h - z; cbt = -cbt; tw = -tw; }
                    else break;
                }
            }
            pz = xclamp(z, zmin, h);
        }
        if (sub < a.n_sub - 1u) hanna_short_cell_t<T>(cell, pz, sigw, dsigwdz, tlw);
    }
}

// Turbulence of one particle in the fused step (langevin_fused.wgsl:414-515
// after the PBL lookup and the noise draws): Hanna at the particle height,
// then turbulence_from_hanna.
template <class T>
__device__ __forceinline__ void turbulence_update(const StepArgs& a, const CellHanna& cell, float2 e_uv,
                                                  float2 e_w01, float2 e_w23, T& pz, T& tu, T& tv, T& tw,
                                                  int32_t& cbt) {
    const HannaT<T> hn = compute_hanna_cell_t<T>(cell, pz);
    turbulence_from_hanna<T, HannaLangevin>(a, cell, hn, e_uv, e_w01, e_w23, pz, tu, tv, tw, cbt);
}

// What the step records for its adjoint (a policy of particle_step): NoTape
// records nothing and keeps the plain float path.
struct NoTape {
    static constexpr bool on = false;
    __device__ __forceinline__ void advect(uint32_t, float, float, float, float, float, float, uint32_t) {}
    __device__ __forceinline__ void turb(uint32_t, float, float, float, float, float, float, float, float) {}
    __device__ __forceinline__ void deposit(uint32_t, float) {}
    __device__ __forceinline__ void out(uint32_t, float, float, float, float) {}
};

// Clamp states of the advection, one bit each: set when the raw value lies
// strictly inside its clamp range (the clamp passes the derivative).
enum : uint32_t { ADV_PX = 1u, ADV_PY = 2u, ADV_PZ = 4u, ADV_X1 = 8u, ADV_Y1 = 16u, ADV_Z1 = 32u };

__device__ __forceinline__ uint32_t inside(float v, float lo, float hi, uint32_t bit) {
    return (v > lo && v < hi) ? bit : 0u;
}

template <class Tape>
__device__ __forceinline__ void particle_step_t(const StepArgs& a, const Levels& lv, uint32_t p,
                                                uint32_t rng_index, float alpha, u32x4 counter, uint32_t key0,
                                                uint32_t key1, Tape& tape) {
    const bool dry_on = (a.stages & FPG_STAGE_DRY) && a.dry_mode != FPG_FORCING_NONE;
    const bool wet_on = (a.stages & FPG_STAGE_WET) && a.wet_mode != FPG_FORCING_NONE;
    if (!(a.flags[p] & FLAG_ACTIVE)) {
        if (dry_on && a.dry_prob) a.dry_prob[p] = 0.0f;
        if (wet_on && a.wet_prob) a.wet_prob[p] = 0.0f;
        return;
    }
    int32_t cx = a.cell_x[p], cy = a.cell_y[p];
    float px = a.pos_x[p], py = a.pos_y[p], pz = a.pos_z[p];
    const bool turb_on = (a.stages & FPG_STAGE_TURBULENCE) != 0;
    float tu = a.turb_u[p], tv = a.turb_v[p];

    // ---- advection_dual_wind.wgsl:266-300 ----
    if (a.stages & FPG_STAGE_ADVECT) {
        const float x0 = (float)cx + px;
        const float y0 = (float)cy + py;
        const float z0 = pz;
        const float3 s0 = sample_dual(a, lv, x0, y0, z0, alpha);
        const float u0 = s0.x + tu, v0 = s0.y + tv, w0 = s0.z;
        const float xmax = (float)(a.nx - 1u), ymax = (float)(a.ny - 1u);
        const float ztop = a.has_heights ? lv.h[a.nz - 1u] : (float)(a.nz - 1u);
        const float rxp = x0 + (u0 * a.xs) * a.dt;
        const float ryp = y0 + (v0 * a.ys) * a.dt;
        const float rzp = z0 + (w0 * a.zs) * a.dt;
        const float pxp = clampf(rxp, 0.0f, xmax);
        const float pyp = clampf(ryp, 0.0f, ymax);
        const float pzp = clampf(rzp, 0.0f, ztop);
        const float3 s1 = sample_dual(a, lv, pxp, pyp, pzp, alpha);
        const float u1 = s1.x + tu, v1 = s1.y + tv, w1 = s1.z;
        const float cu = 0.5f * (u0 + u1), cv = 0.5f * (v0 + v1), cw = 0.5f * (w0 + w1);
        const float rx1 = x0 + (cu * a.xs) * a.dt;
        const float ry1 = y0 + (cv * a.ys) * a.dt;
        const float rz1 = z0 + (cw * a.zs) * a.dt;
        const float x1 = clampf(rx1, 0.0f, xmax);
        const float y1 = clampf(ry1, 0.0f, ymax);
        pz = clampf(rz1, 0.0f, ztop);
        if constexpr (Tape::on) {
            const uint32_t fl = inside(rxp, 0.0f, xmax, ADV_PX) | inside(ryp, 0.0f, ymax, ADV_PY) |
                                inside(rzp, 0.0f, ztop, ADV_PZ) | inside(rx1, 0.0f, xmax, ADV_X1) |
                                inside(ry1, 0.0f, ymax, ADV_Y1) | inside(rz1, 0.0f, ztop, ADV_Z1);
            tape.advect(p, x0, y0, z0, pxp, pyp, pzp, fl);
        }
        split_coord(x1, a.nx, cx, px);
        split_coord(y1, a.ny, cy, py);
        a.cell_x[p] = cx; a.cell_y[p] = cy;
        a.pos_x[p] = px; a.pos_y[p] = py;
        a.vel_u[p] = cu; a.vel_v[p] = cv; a.vel_w[p] = cw;
    }

    // ---- langevin_fused.wgsl:414-515 ----
    if (turb_on) {
        const float x = (float)cx + px;
        const float y = (float)cy + py;
        const uint32_t i = (uint32_t)floorf(clampf(x, 0.0f, (float)(a.pnx - 1u)));
        const uint32_t j = (uint32_t)floorf(clampf(y, 0.0f, (float)(a.pny - 1u)));
        const CellHanna cell = ld_cell_hanna(a.hcell + (i * a.pny + j));

        const uint32_t n_vert = a.n_sub > 1u ? a.n_sub : 1u;
        const uint32_t blocks = (2u + n_vert + 3u) / 4u;
        const u32x4 b0 = philox4x32_10(counter_add(counter, rng_index * blocks), key0, key1);
        u32x4 b1 = {0u, 0u, 0u, 0u};
        if (blocks > 1u) b1 = philox4x32_10(counter_add(counter, rng_index * blocks + 1u), key0, key1);
        const float2 e_uv = box_muller(u32_to_uniform01(b0.x), u32_to_uniform01(b0.y));
        const float2 e_w01 = box_muller(u32_to_uniform01(b0.z), u32_to_uniform01(b0.w));
        const float2 e_w23 = box_muller(u32_to_uniform01(b1.x), u32_to_uniform01(b1.y));

        float tw = a.turb_w[p];
        const int32_t cbt_in = a.n_sub == 0u ? 0 : a.cbt[p];
        int32_t cbt = cbt_in;
        if constexpr (Tape::on) {
            // tangents: .a along the height after advection (and, for tu/tv,
            // .b along their own input); .b of z and tw along the input tw
            D2 zd(pz, 1.0f, 0.0f), ud(tu, 0.0f, 1.0f), vd(tv, 0.0f, 1.0f), wd(tw, 0.0f, 1.0f);
            turbulence_update<D2>(a, cell, e_uv, e_w01, e_w23, zd, ud, vd, wd, cbt);
            tape.turb(p, zd.a, zd.b, wd.a, wd.b, ud.a, ud.b, vd.a, vd.b);
            pz = zd.v; tu = ud.v; tv = vd.v; tw = wd.v;
        } else {
            turbulence_update<float>(a, cell, e_uv, e_w01, e_w23, pz, tu, tv, tw, cbt);
        }
        if (a.n_sub != 0u && cbt != cbt_in) a.cbt[p] = cbt;
        a.turb_u[p] = tu; a.turb_v[p] = tv; a.turb_w[p] = tw;
    }
    if ((a.stages & FPG_STAGE_ADVECT) || (turb_on && a.n_sub != 0u)) a.pos_z[p] = pz;

    // ---- dry_deposition.wgsl:89-105 and wet_deposition.wgsl:203-216 ----
    float surv_total = 1.0f;
    if (dry_on || wet_on) {
        float survival = 1.0f;
        if (dry_on) {
            float prob = 0.0f;
            if (!(pz >= 2.0f * a.href)) {
                const float vd = a.dry_mode == FPG_FORCING_PER_PARTICLE ? a.dry_v_arr[p] : a.dry_v;
                const float s = dry_survival(vd, a.tdt, a.href);
                prob = 1.0f - s;
                survival = s;
            }
            if (a.dry_prob) a.dry_prob[p] = prob;
        }
        float wsurv = 1.0f;
        if (wet_on) {
            float lam, fr;
            if (a.wet_mode == FPG_FORCING_PER_PARTICLE) {
                lam = a.wet_l_arr[p]; fr = a.wet_f_arr[p];
            } else if (a.wet_mode == FPG_FORCING_PER_CELL) {
                const float x = (float)cx + px;
                const float y = (float)cy + py;
                const uint32_t i = (uint32_t)floorf(clampf(x, 0.0f, (float)(a.wnx - 1u)));
                const uint32_t j = (uint32_t)floorf(clampf(y, 0.0f, (float)(a.wny - 1u)));
                const float2 c = __ldg(a.wet_cells + (i * a.wny + j));
                lam = c.x; fr = c.y;
            } else {
                lam = a.wet_l; fr = a.wet_f;
            }
            const float prob = wet_probability(lam, a.tdt, fr);
            wsurv = 1.0f - prob;
            if (a.wet_prob) a.wet_prob[p] = prob;
        }
        // mass * dry survival, then * wet survival: two roundings, as the
        // two reference passes apply them.
        for (int k = 0; k < a.n_species; ++k) {
            float m = a.mass[k][p];
            if (dry_on && !(pz >= 2.0f * a.href)) m = m * survival;
            if (wet_on) m = m * wsurv;
            a.mass[k][p] = m;
        }
        if constexpr (Tape::on) surv_total = (dry_on && !(pz >= 2.0f * a.href) ? survival : 1.0f) * wsurv;
    }
    if constexpr (Tape::on) {
        tape.deposit(p, surv_total);
        tape.out(p, (float)cx + px, (float)cy + py, pz, a.mass[0][p]);
    }
}

__device__ __forceinline__ void particle_step(const StepArgs& a, const Levels& lv, uint32_t p,
                                              uint32_t rng_index, float alpha, u32x4 counter, uint32_t key0,
                                              uint32_t key1) {
    NoTape t;
    particle_step_t<NoTape>(a, lv, p, rng_index, alpha, counter, key0, key1, t);
}


__device__ __forceinline__ float sp_(float v, float fb) { return (finitef(v) && v > 0.0f) ? v : fb; }
__device__ __forceinline__ float snn_(float v, float fb) { return (finitef(v) && v >= 0.0f) ? v : fb; }
__device__ __forceinline__ float sf_(float v, float fb) { return finitef(v) ? v : fb; }

// interpolate_surface_fields_linear (io/temporal.rs:99-104,122-214) followed
// by pbl_diagnostics.wgsl:238-305 for one cell.
// interpolate_surface_fields_linear (io/temporal.rs:99-104,122-214) followed by
// pbl_diagnostics.wgsl:238-305 for met cell c.
__device__ __forceinline__ void pbl_cell(const fpg_surface_cell* __restrict__ s0,
                                         const fpg_surface_cell* __restrict__ s1, float alpha,
                                         const fpg_pbl_options& o, uint32_t c, float* ustar_o, float* wstar_o,
                                         float* hmix_o, float* oli_o, float* sshf_o, float* ssr_o,
                                         float* surfstr_o, float4* packed, CellHanna* hanna) {
    float in[10];
    const float* a = &s0[c].surface_pressure_pa;
    const float* b = &s1[c].surface_pressure_pa;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        if (alpha <= 0.0f) in[k] = a[k];
        else if (alpha >= 1.0f) in[k] = b[k];
        else in[k] = lerpf(a[k], b[k], alpha);
    }
    const float sp = in[0], t2 = in[1], u10 = in[2], v10 = in[3], stress = in[4], shf = in[5], ssr = in[6];
    const float hm = in[7], fv = in[8], oli_in = in[9];
    const float temp_k = sp_(t2, 300.0f);
    const float pressure = sp_(sp, 101325.0f);
    const float air_density = pressure / (287.05f * temp_k);
    float est;
    {
        const float rho = sp_(air_density, 1.225f);
        const float safe_stress = snn_(stress, 0.0f);
        if (safe_stress > 0.0f) {
            est = fmaxf(sqrtf(safe_stress / rho), 1.0e-4f);
        } else {
            const float z0 = sp_(o.roughness_length_m, 0.1f);
            const float zr = fmaxf(sp_(o.wind_reference_height_m, 10.0f), 1.01f * z0);
            const float ws = fmaxf(sqrtf(u10 * u10 + v10 * v10), 0.0f);
            if (ws <= 0.0f) {
                est = 1.0e-4f;
            } else {
                const float us = 0.4f * ws / fmaxf(logf(zr / z0), 1.0e-6f);
                est = fmaxf(sp_(us, 1.0e-4f), 1.0e-4f);
            }
        }
    }
    const float ustar = (finitef(fv) && fv > 0.0f) ? fmaxf(fv, 1.0e-4f) : fmaxf(est, 1.0e-4f);
    float computed_ol;
    {
        const float hf = sf_(shf, 0.0f);
        if (fabsf(hf) < fmaxf(o.heat_flux_neutral_threshold_w_m2, 0.0f)) {
            computed_ol = __int_as_float(0x7f800000);
        } else {
            const float u = fmaxf(sp_(ustar, 1.0e-4f), 1.0e-4f);
            const float t = sp_(temp_k, 300.0f);
            const float d = sp_(air_density, 1.225f);
            const float numerator = -(d * 1004.6f * t * u * u * u);
            const float denominator = 0.4f * 9.81f * hf;
            if (fabsf(denominator) < 1.0e-9f) {
                computed_ol = __int_as_float(0x7f800000);
            } else {
                const float olv = numerator / denominator;
                computed_ol = (!finitef(olv) || fabsf(olv) > 1.0e9f) ? __int_as_float(0x7f800000) : olv;
            }
        }
    }
    float oli;
    if (finitef(oli_in) && fabsf(oli_in) >= 1.0e-5f) oli = oli_in;
    else oli = (!finitef(computed_ol) || fabsf(computed_ol) > 1.0e5f) ? 0.0f : 1.0f / computed_ol;
    const float hsrc = (finitef(hm) && hm > 0.0f) ? hm : o.fallback_mixing_height_m;
    const float hmix = fmaxf(clampf(hsrc, o.hmix_min_m, o.hmix_max_m), o.hmix_min_m);
    const float safe_shf = sf_(shf, 0.0f);
    float wstar = 0.0f;
    if (safe_shf > 0.0f) {
        const float d = sp_(air_density, 1.225f);
        const float t = sp_(temp_k, 300.0f);
        const float hh = sp_(hmix, o.hmix_min_m);
        const float bf = safe_shf / (d * 1004.6f) * 9.81f / t;
        if (!(bf <= 0.0f || !finitef(bf))) wstar = fmaxf(powf(bf * hh, 1.0f / 3.0f), 0.0f);
    }
    ustar_o[c] = ustar; wstar_o[c] = wstar; hmix_o[c] = hmix; oli_o[c] = oli;
    sshf_o[c] = sf_(shf, 0.0f);
    ssr_o[c] = snn_(ssr, 0.0f);
    surfstr_o[c] = snn_(stress, 0.0f);
    packed[c] = make_float4(ustar, wstar, hmix, oli);
    st_cell_hanna(hanna + c, cell_hanna(ustar, wstar, obukhov_from_inverse(oli), hmix));
}

__device__ __forceinline__ float snn0(float v) { return (finitef(v) && v > 0.0f) ? v : 0.0f; }
__device__ __forceinline__ int precip_class(float p) {
    return p > 20.0f ? 4 : p > 8.0f ? 3 : p > 3.0f ? 2 : p > 1.0f ? 1 : 0;
}

// wet_precipitation_state + below_cloud_scavenging_coefficient_gas
// (physics/wet_scavenging.rs:179-225,78-82) for one met cell: (lambda, fraction).
__device__ __forceinline__ float2 wet_cell_forcing(float lsp_in, float conv_in, float cc_in, float a_in,
                                                   float b_in) {
    const float lsf[5] = {0.5f, 0.65f, 0.8f, 0.9f, 0.95f};
    const float cvf[5] = {0.4f, 0.55f, 0.7f, 0.8f, 0.9f};
    const float lsp = snn0(lsp_in), convp = snn0(conv_in);
    const float total = lsp + convp;
    float fraction = 0.0f, subgrid = 0.0f;
    if (!(total < 0.01f)) {
        const float cc = clampf(cc_in, 0.0f, 1.0f);
        const float weighted = (lsp * lsf[precip_class(lsp)] + convp * cvf[precip_class(convp)]) / fmaxf(total, 1.0e-12f);
        const float area = fminf(fmaxf(fmaxf(cc * weighted, 0.05f), 0.05f), 1.0f);
        subgrid = snn0(total / fmaxf(area, 1.0e-12f));
        fraction = area;
    }
    float lambda = 0.0f;
    if (total >= 0.01f && fraction > 0.0f && subgrid > 0.0f) {
        lambda = snn0(snn0(a_in) * powf(subgrid, snn0(b_in)));
    } else {
        fraction = 0.0f;
    }
    return make_float2(lambda, fraction);
}

}  // namespace fpg
