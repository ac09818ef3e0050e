// physics.cuh — per-particle device physics of the flexpart-gpu step.
//
// One __device__ function per reference routine, each citing the WGSL shader
// (the reference GPU path) and the Rust CPU routine it restates.  All code is
// compiled with -fmad=false: every multiply and add rounds separately, exactly
// as written, and the only fused operation is the explicit fmaf of lerp()
// (the reference CPU lerp is `a.mul_add(1 - t, b * t)`,
// src/physics/interpolation.rs:75-77, src/io/temporal.rs:417-420).
// Transcendentals: cbrtf and expf (deposition) as CUDA computes them; the
// Hanna and Langevin exponentials and powers at the accuracy WGSL specifies
// for the reference's shaders (__expf, __powf); the Box-Muller logarithm,
// sine and cosine of box_muller_math.h.  sqrtf is correctly rounded, and
// '/' is too except in the step's units (step.cu, batch.cu, adjoint.cu),
// which the build compiles with the approximate full-range division (within
// 2 ulp) and with subnormal values flushed to zero.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "box_muller_math.h"

namespace fpg {

constexpr uint32_t FLAG_ACTIVE = 1u;

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ bool finitef(float v) { return isfinite(v); }
__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(a, 1.0f - t, b * t); }
__device__ __forceinline__ float sanitize_positive(float v) { return (finitef(v) && v > 0.0f) ? v : 0.0f; }

// The division of the per-particle step.  The step's units are built with
// FPG_RECIPROCAL_DIVISION: a / b is then a times the approximate reciprocal
// of b (__fdividef), within 2 ulp for |b| in [2^-126, 2^126] -- the range
// over which WGSL specifies x / y, to 2.5 ULP, for the reference's shaders --
// and there the same bits as the approximate full-range division
// (-prec-div=false; equal on 16.8 M random pairs with b in [1e-4, 1e5]) in
// two instructions fewer.  The step divides by heights, velocity scales,
// Lagrangian time scales and the Obukhov length, all inside that range.
// Other units divide in IEEE arithmetic.
__device__ __forceinline__ float sdiv(float a, float b) {
#ifdef FPG_RECIPROCAL_DIVISION
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
__device__ __forceinline__ float xdiv(float a, float b) { return sdiv(a, b); }

// x^(1/3), x^(2/3) and x^(-1/3) for x >= 0 from one cbrtf (max 1 ulp): the
// reference writes pow(x, 1.0/3.0), pow(x, 2.0/3.0), pow(x, -1.0/3.0)
// (hanna.rs:81-92, langevin_fused.wgsl:247-254,315-321).  The results stay
// within a few ulp of powf with the f32-rounded exponents (1/3 rounds to
// 0.33333334, a relative exponent error of 3e-8), at a fraction of its cost.
__device__ __forceinline__ float pow_third(float x) { return cbrtf(x); }

// ---- Philox4x32-10 (src/physics/rng.rs:28-65, langevin_fused.wgsl:126-169) --
struct u32x4 { uint32_t x, y, z, w; };

__device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// counter_add with a u32 offset (langevin_fused.wgsl:171-180).
__device__ __forceinline__ u32x4 counter_add(u32x4 b, uint32_t offset) {
    u32x4 r;
    r.x = b.x + offset;
    const uint32_t c0 = r.x < b.x;
    r.y = b.y + c0;
    const uint32_t c1 = (c0 == 1u) && (r.y < b.y);
    r.z = b.z + c1;
    const uint32_t c2 = (c1 == 1u) && (r.z < b.z);
    r.w = b.w + c2;
    return r;
}

// u32_to_uniform01 (rng.rs:94-96).
__device__ __forceinline__ float u32_to_uniform01(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

// box_muller_normals (physics/langevin.rs:176-182, langevin_fused.wgsl:186-192),
// with the logarithm and the sine and cosine of box_muller_math.h: written
// for these inputs (u0 in {FLT_MIN} and [2^-24, 1 - 2^-24], theta = 2pi u1
// in [0, 2pi)), within 1.5 ulp of the exact values, and closer to the libm
// results of the reference's CPU path than CUDA's logf and sincosf.
__device__ __forceinline__ float2 box_muller(float u0, float u1) {
    const float ru = clampf(u0, 1.17549435e-38f, 0.99999994f);
    const float au = clampf(u1, 0.0f, 0.99999994f);
    const float radius = sqrtf(-2.0f * bm_log(ru));
    const float theta = 6.2831855f * au;
    float sn, cs;
    bm_sincos(theta, &sn, &cs);
    return make_float2(radius * cs, radius * sn);
}

// ---- scalar helpers of the templated physics --------------------------------
// The Hanna and Langevin routines below are templates over the scalar type:
// float for the step itself, and the dual number of the adjoint (dual.cuh),
// which carries derivatives beside the value and supplies the same helper
// names.  For float every helper is the plain CUDA call, so the float
// instantiation performs exactly the operations written, in the same order.
//
// The exponentials and powers of the Hanna profiles and the Langevin updates
// run at the accuracy WGSL specifies for the reference's shaders, which
// compute them (langevin_fused.wgsl:224-389): exp within 3 + 2|x| ulp, pow
// inherited from exp2(y log2 x).  CUDA's __expf stays within 2 +
// floor(1.173|x|) ulp and __powf is exp2 of y times the hardware log2, the
// same construction as WGSL's pow; both cost a few instructions where expf
// and powf cost 9 and about 30, and a particle-step takes up to seven
// exponentials and four powers.
__device__ __forceinline__ float val(float x) { return x; }
__device__ __forceinline__ float xexp(float x) { return __expf(x); }
__device__ __forceinline__ float xsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ float xcbrt(float x) { return pow_third(x); }
// x^e for x > 0 by __powf: the reference's pow(zeta, 0.8) of the
// stable-branch T_L (hanna.rs:111, langevin_fused.wgsl:271,332).  x <= 0
// goes to powf (0^0.8 = 0).
__device__ __forceinline__ float pow_pos(float x, float e) { return x > 0.0f ? __powf(x, e) : powf(x, e); }
__device__ __forceinline__ float xpow(float x, float e) { return pow_pos(x, e); }
__device__ __forceinline__ float xmax(float x, float c) { return fmaxf(x, c); }
__device__ __forceinline__ float xclamp(float x, float lo, float hi) { return clampf(x, lo, hi); }
__device__ __forceinline__ float xabs(float x) { return fabsf(x); }

// ---- Hanna (physics/hanna.rs:49-163, langevin_fused.wgsl:224-293) ----------
// Stability branch of hanna.rs:69-112: 0 neutral, 1 unstable, 2 stable.
enum { REGIME_NEUTRAL = 0, REGIME_UNSTABLE = 1, REGIME_STABLE = 2 };

template <class T>
struct HannaT {
    float ust, wst, ol, h;
    T sigu, sigv, sigw, dsigwdz, tlu, tlv, tlw;
    int regime;
};
using Hanna = HannaT<float>;

__device__ __forceinline__ float obukhov_from_inverse(float oli) {
    // hanna.rs:169-174: |1/L| < 1e-5 is neutral (L = +inf).
    return fabsf(oli) < 1.0e-5f ? __int_as_float(0x7f800000) : 1.0f / oli;
}

__device__ __forceinline__ int hanna_regime(float ol, float h) {
    return (!finitef(ol) || ol == 0.0f || h / fabsf(ol) < 1.0f) ? REGIME_NEUTRAL
           : ol < 0.0f                                         ? REGIME_UNSTABLE
                                                               : REGIME_STABLE;
}

// ---- per-cell Hanna constants -----------------------------------------------
// What compute_hanna and hanna_short_w derive from a met cell's PBL
// parameters alone, computed once per cell (pbl_cell) instead of up to four
// times per particle-step: the floored u*, w*, h (hanna.rs:50-53), the
// Obukhov length, the stability regime, and per regime
//   * the leading constant factors of the reference's products, which C++
//     evaluates left to right (1.2f * wst * wst * (1 - 0.9 zeta) * z23
//     rounds (1.2f * wst) * wst first), so the per-cell product is the same
//     float the per-particle expression forms;
//   * the outputs that depend on the cell only, floored and sanitised as
//     compute_hanna does: sigma_u = sigma_v and T_Lu = T_Lv of the unstable
//     branch (hanna.rs:81-86, 120-131), dsigma_w/dz of the stable branch
//     (hanna.rs:106).
// Same operations in the same order: the per-particle results are bit for
// bit those of evaluating everything per particle.
//   neutral:  k0 = 2 u*,  k1 = 1.3 u*
//   unstable: k0 = sigma_u, k1 = T_Lu, k2 = 1.2 w* w*, k3 = -1.4 u* u*,
//             k4 = w* w*, k5 = 0.15 h
//   stable:   k0 = 2 u*,  k1 = 1.3 u*, k2 = dsigma_w/dz, k5 = 0.15 h, k6 = 0.1 h
struct __align__(16) CellHanna {
    float ust, wst, h, ol;
    float k0, k1, k2, k3;
    float k4, k5, k6;
    int regime;
};

// The constants of `regime` for a cell (ust, wst, h unfloored; ol = L).
__device__ __forceinline__ CellHanna cell_hanna_for_regime(float ust_in, float wst_in, float ol, float h_in,
                                                           int regime) {
    CellHanna c;
    c.ust = fmaxf(ust_in, 1.0e-4f);
    c.wst = fmaxf(wst_in, 0.0f);
    c.h = fmaxf(h_in, 1.0f);
    c.ol = ol;
    c.regime = regime;
    c.k0 = c.k1 = c.k2 = c.k3 = c.k4 = c.k5 = c.k6 = 0.0f;
    if (regime == REGIME_UNSTABLE) {
        float sigu = 1.0e-2f + c.ust * pow_third(12.0f - 0.5f * c.h / ol);
        float tlu = 0.15f * c.h / sigu;
        tlu = fmaxf(tlu, 10.0f);
        if (!finitef(sigu) || sigu <= 0.0f) sigu = 1.0e-2f;
        if (!finitef(tlu)) tlu = 10.0f;
        c.k0 = sigu;
        c.k1 = tlu;
        c.k2 = 1.2f * c.wst * c.wst;
        c.k3 = -1.4f * c.ust * c.ust;
        c.k4 = c.wst * c.wst;
        c.k5 = 0.15f * c.h;
    } else {
        c.k0 = 2.0f * c.ust;
        c.k1 = 1.3f * c.ust;
        if (regime == REGIME_STABLE) {
            float d = -1.3f * c.ust / c.h;
            if (d == 0.0f) d = 1.0e-10f;
            if (!finitef(d)) d = 1.0e-10f;
            c.k2 = d;
            c.k5 = 0.15f * c.h;
            c.k6 = 0.1f * c.h;
        }
    }
    return c;
}

// The constants of a cell's own regime (the branch test of hanna.rs:69-112
// on the floored h).
__device__ __forceinline__ CellHanna cell_hanna(float ust_in, float wst_in, float ol, float h_in) {
    return cell_hanna_for_regime(ust_in, wst_in, ol, h_in, hanna_regime(ol, fmaxf(h_in, 1.0f)));
}

__device__ __forceinline__ CellHanna ld_cell_hanna(const CellHanna* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = __ldg(q), b = __ldg(q + 1), d = __ldg(q + 2);
    CellHanna c;
    c.ust = a.x; c.wst = a.y; c.h = a.z; c.ol = a.w;
    c.k0 = b.x; c.k1 = b.y; c.k2 = b.z; c.k3 = b.w;
    c.k4 = d.x; c.k5 = d.y; c.k6 = d.z; c.regime = __float_as_int(d.w);
    return c;
}

__device__ __forceinline__ void st_cell_hanna(CellHanna* p, const CellHanna& c) {
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(c.ust, c.wst, c.h, c.ol);
    q[1] = make_float4(c.k0, c.k1, c.k2, c.k3);
    q[2] = make_float4(c.k4, c.k5, c.k6, __int_as_float(c.regime));
}

// sigma_w, dsigma_w/dz, T_Lw of the unstable branch at height z
// (hanna.rs:87-104,132-141, langevin_fused.wgsl:305-327).
template <class T>
__device__ __forceinline__ void hanna_unstable_w(const CellHanna& c, T z, T zeta, T& sigw, T& dsigwdz, T& tlw) {
    const T cz = xcbrt(zeta);
    const T z23 = cz * cz;
    const T sigw_sq = c.k2 * (1.0f - 0.9f * zeta) * z23 + (1.8f - 1.4f * zeta) * c.ust * c.ust;
    sigw = xsqrt(sigw_sq) + 1.0e-2f;
    const T zm13 = xdiv(1.0f, (val(zeta) >= 1.0e-3f ? cz : T(pow_third(1.0e-3f))));
    dsigwdz = xdiv(xdiv(0.5f, sigw), c.h) * (c.k3 + c.k4 * (0.8f * zm13 - 1.8f * z23));
    if (val(z) < fabsf(c.ol)) tlw = xdiv(0.1f * z, sigw * (0.55f - 0.38f * xabs(xdiv(z, c.ol))));
    else if (val(zeta) < 0.1f) tlw = xdiv(0.59f * z, sigw);
    else tlw = xdiv(c.k5, sigw) * (1.0f - xexp(-5.0f * zeta));
}

// compute_hanna_params (physics/hanna.rs:49-163) at height z_in of a cell.
template <class T>
__device__ __forceinline__ HannaT<T> compute_hanna_cell_t(const CellHanna& c, T z_in) {
    HannaT<T> o;
    const float ust = c.ust, h = c.h;
    const T z = xclamp(z_in, 0.0f, h);
    const T zeta = xclamp(xdiv(z, h), 0.0f, 1.0f);
    T sigu, sigv, sigw, dsigwdz, tlu, tlv, tlw;
    o.regime = c.regime;
    if (c.regime == REGIME_NEUTRAL) {
        const T corr = xdiv(z, ust);
        sigu = 1.0e-2f + c.k0 * xexp(-3.0e-4f * corr);
        sigw = c.k1 * xexp(-2.0e-4f * corr);
        dsigwdz = -2.0e-4f * sigw;
        sigw = sigw + 1.0e-2f;
        sigv = sigw;
        tlu = xdiv(xdiv(0.5f * z, sigw), (1.0f + 1.5e-3f * corr));
        tlv = tlu;
        tlw = tlu;
        tlu = xmax(tlu, 10.0f);
        tlv = xmax(tlv, 10.0f);
        tlw = xmax(tlw, 30.0f);
        if (val(dsigwdz) == 0.0f) dsigwdz = T(1.0e-10f);
        if (!finitef(val(sigu)) || val(sigu) <= 0.0f) sigu = T(1.0e-2f);
        if (!finitef(val(sigv)) || val(sigv) <= 0.0f) sigv = T(1.0e-2f);
        if (!finitef(val(sigw)) || val(sigw) <= 0.0f) sigw = T(1.0e-2f);
        if (!finitef(val(tlu))) tlu = T(10.0f);
        if (!finitef(val(tlv))) tlv = T(10.0f);
        if (!finitef(val(tlw))) tlw = T(30.0f);
        if (!finitef(val(dsigwdz))) dsigwdz = T(1.0e-10f);
    } else if (c.regime == REGIME_UNSTABLE) {
        // sigma_u, sigma_v, T_Lu, T_Lv: the cell's, already final
        sigu = T(c.k0);
        sigv = sigu;
        tlu = T(c.k1);
        tlv = tlu;
        hanna_unstable_w<T>(c, z, zeta, sigw, dsigwdz, tlw);
        tlw = xmax(tlw, 30.0f);
        if (val(dsigwdz) == 0.0f) dsigwdz = T(1.0e-10f);
        if (!finitef(val(sigw)) || val(sigw) <= 0.0f) sigw = T(1.0e-2f);
        if (!finitef(val(tlw))) tlw = T(30.0f);
        if (!finitef(val(dsigwdz))) dsigwdz = T(1.0e-10f);
    } else {
        sigu = 1.0e-2f + c.k0 * (1.0f - zeta);
        sigv = 1.0e-2f + c.k1 * (1.0f - zeta);
        sigw = sigv;
        dsigwdz = T(c.k2);                       // the cell's, already final
        tlu = xdiv(c.k5, sigu) * xsqrt(zeta);
        tlv = 0.467f * tlu;
        tlw = xdiv(c.k6, sigw) * xpow(zeta, 0.8f);
        tlu = xmax(tlu, 10.0f);
        tlv = xmax(tlv, 10.0f);
        tlw = xmax(tlw, 30.0f);
        if (!finitef(val(sigu)) || val(sigu) <= 0.0f) sigu = T(1.0e-2f);
        if (!finitef(val(sigv)) || val(sigv) <= 0.0f) sigv = T(1.0e-2f);
        if (!finitef(val(sigw)) || val(sigw) <= 0.0f) sigw = T(1.0e-2f);
        if (!finitef(val(tlu))) tlu = T(10.0f);
        if (!finitef(val(tlv))) tlv = T(10.0f);
        if (!finitef(val(tlw))) tlw = T(30.0f);
    }
    o.ust = c.ust; o.wst = c.wst; o.ol = c.ol; o.h = c.h;
    o.sigu = sigu; o.sigv = sigv; o.sigw = sigw; o.dsigwdz = dsigwdz;
    o.tlu = tlu; o.tlv = tlv; o.tlw = tlw;
    return o;
}

template <class T>
__device__ __forceinline__ HannaT<T> compute_hanna_t(float ust_in, float wst_in, float ol, float h_in, T z_in) {
    return compute_hanna_cell_t<T>(cell_hanna(ust_in, wst_in, ol, h_in), z_in);
}

__device__ __forceinline__ Hanna compute_hanna(float ust_in, float wst_in, float ol, float h_in, float z_in) {
    return compute_hanna_t<float>(ust_in, wst_in, ol, h_in, z_in);
}

// hanna_short_w (langevin_fused.wgsl:296-344): sigw, dsigwdz, tlw at a new
// height in a cell.  The shader's branch test (`!finite(ol) || ol == 0 ||
// h/|ol| < 1`, then `ol < 0`) sees the same floored h and the same ol as
// compute_hanna's for this particle, so its outcome is the cell's regime.
template <class T>
__device__ __forceinline__ void hanna_short_cell_t(const CellHanna& c, T z_in, T& sigw_o, T& dsigwdz_o, T& tlw_o) {
    const T z = xclamp(z_in, 0.0f, c.h);
    const T zeta = xclamp(xdiv(z, c.h), 0.0f, 1.0f);
    T sigw, dsigwdz, tlw;
    if (c.regime == REGIME_NEUTRAL) {
        const T corr = xdiv(z, c.ust);
        sigw = c.k1 * xexp(-2.0e-4f * corr);
        dsigwdz = -2.0e-4f * sigw;
        sigw = sigw + 1.0e-2f;
        tlw = xdiv(xdiv(0.5f * z, sigw), (1.0f + 1.5e-3f * corr));
    } else if (c.regime == REGIME_UNSTABLE) {
        hanna_unstable_w<T>(c, z, zeta, sigw, dsigwdz, tlw);
    } else {
        sigw = 1.0e-2f + c.k1 * (1.0f - zeta);
        dsigwdz = T(c.k2);                       // the cell's, already final
        tlw = xdiv(c.k6, sigw) * xpow(zeta, 0.8f);
    }
    tlw = xmax(tlw, 30.0f);
    if (c.regime != REGIME_STABLE) {
        if (val(dsigwdz) == 0.0f) dsigwdz = T(1.0e-10f);
        if (!finitef(val(dsigwdz))) dsigwdz = T(1.0e-10f);
    }
    if (!finitef(val(sigw)) || val(sigw) <= 0.0f) sigw = T(1.0e-2f);
    if (!finitef(val(tlw))) tlw = T(30.0f);
    sigw_o = sigw; dsigwdz_o = dsigwdz; tlw_o = tlw;
}

// The same from a cell's raw parameters with the branch given by the caller
// (ust, wst, h floored here, as hanna_short_w receives them).
template <class T>
__device__ __forceinline__ void hanna_short_w_t(float ust_in, float wst_in, float ol, float h_in, T z_in, int regime,
                                                T& sigw_o, T& dsigwdz_o, T& tlw_o) {
    hanna_short_cell_t<T>(cell_hanna_for_regime(ust_in, wst_in, ol, h_in, regime), z_in, sigw_o, dsigwdz_o, tlw_o);
}

__device__ __forceinline__ void hanna_short_w(float ust_in, float wst_in, float ol, float h_in, float z_in,
                                              int regime, float& sigw_o, float& dsigwdz_o, float& tlw_o) {
    hanna_short_w_t<float>(ust_in, wst_in, ol, h_in, z_in, regime, sigw_o, dsigwdz_o, tlw_o);
}

// The Langevin updates below take Hanna outputs only: sigma >= 0.01 and
// T_L >= 10 s (30 s vertical), both finite after the clamps above, so the
// reference's sanitize_positive() and its T_L == 0 return
// (physics/langevin.rs:116-121,146-150) are the identity and are omitted.

// ---- Langevin OU updates (physics/langevin.rs:116-170, langevin_fused.wgsl:350-389)
template <class T>
__device__ __forceinline__ T langevin_h_t(T prev, T sigma, T tl, float dt, float eta) {
    const T ratio = xdiv(dt, tl);
    T next;
    if (val(ratio) < 0.5f) {
        next = (1.0f - ratio) * prev + eta * sigma * xsqrt(xmax(2.0f * ratio, 0.0f));
    } else {
        const T corr = xexp(-ratio);
        next = corr * prev + eta * sigma * xsqrt(xmax(1.0f - corr * corr, 0.0f));
    }
    return finitef(val(next)) ? next : T(0.0f);
}

template <class T>
__device__ __forceinline__ T langevin_v_t(T prev, T sigma_w, T tlw, T dsigwdz, float dt, float rho, float eta) {
    const T drift = sigma_w * (dsigwdz + rho * sigma_w);
    const T ratio = xdiv(dt, tlw);
    T next;
    if (val(ratio) < 0.5f) {
        next = (1.0f - ratio) * prev + eta * sigma_w * xsqrt(xmax(2.0f * ratio, 0.0f)) + dt * drift;
    } else {
        const T corr = xexp(-ratio);
        next = corr * prev + eta * sigma_w * xsqrt(xmax(1.0f - corr * corr, 0.0f)) + tlw * (1.0f - corr) * drift;
    }
    return finitef(val(next)) ? next : T(0.0f);
}

__device__ __forceinline__ float langevin_h(float prev, float sigma, float tl, float dt, float eta) {
    return langevin_h_t<float>(prev, sigma, tl, dt, eta);
}

__device__ __forceinline__ float langevin_v(float prev, float sigma_w, float tlw, float dsigwdz, float dt,
                                            float rho, float eta) {
    return langevin_v_t<float>(prev, sigma_w, tlw, dsigwdz, dt, rho, eta);
}

// ---- Deposition --------------------------------------------------------------
// dry_deposition.wgsl:70-74 (survival factor; href already floored at 0.1 m).
__device__ __forceinline__ float dry_survival(float vdep, float dt, float href) {
    const float exponent = sdiv(-fmaxf(vdep, 0.0f) * fabsf(dt), 2.0f * href);
    return clampf(expf(exponent), 0.0f, 1.0f);
}

// wet_deposition.wgsl:179-188, physics/wet_scavenging.rs:375-384.
__device__ __forceinline__ float wet_probability(float lambda_in, float dt_in, float fraction_in) {
    const float lambda = fmaxf(lambda_in, 0.0f);
    const float dt = fabsf(dt_in);
    const float fraction = clampf(fraction_in, 0.0f, 1.0f);
    if (lambda <= 0.0f || dt <= 0.0f || fraction <= 0.0f) return 0.0f;
    const float local = 1.0f - expf(-lambda * dt);
    return clampf(local * fraction, 0.0f, 1.0f);
}

}  // namespace fpg
