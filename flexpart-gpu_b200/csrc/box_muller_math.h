// box_muller_math.h -- the logarithm and the sine and cosine of the
// Box-Muller draws (box_muller_normals, physics/langevin.rs:176-182,
// langevin_fused.wgsl:186-192), written for the inputs the step gives them:
// ln u for u in {FLT_MIN} and [2^-24, 1 - 2^-24] (the clamped 24-bit
// uniforms), sin and cos of theta = 2pi u for u in [0, 1 - 2^-24].
//
//   ln:  u = m 2^e with m in [1/sqrt2, sqrt2) (an integer split of the
//        exponent), f = m - 1 (exact), ln(1 + f) = f + f^2 Q(f) with Q a
//        degree-8 near-minimax polynomial of the relative error on
//        [1/sqrt2 - 1, sqrt2 - 1], then e ln2 added in two parts (ln2_hi has
//        16 significant bits, so e ln2_hi is exact).
//   sin, cos: Cody-Waite reduction r = theta - q pi/2 with pi/2 in three
//        parts and fused multiply-adds (the first step is exact for
//        theta < 2pi), r in [-pi/4, pi/4]; sin r = r + r^3 S(r^2) and
//        cos r = 1 - (r^2/2 - r^4 C(r^2)) with S and C of degree 2; then the
//        quadrant q.
//
// The polynomials were fitted by Lawson's iteratively reweighted least
// squares (box_muller_fit.py) and rounded to float.  Every operation is an
// IEEE single-precision multiply, add or fused multiply-add (the step's
// units compile with -fmad=false; the products that should fuse are
// written as fmaf), so host and device compute the same bits.  Over every
// input the step can give them the error is at most 0.87 ulp (ln), 1.50 ulp
// (sin) and 1.48 ulp (cos), and the results equal glibc's logf, sinf and
// cosf on 92.9 %, 87.0 % and 81.7 % of the inputs (CUDA's logf and sincosf:
// 92.1 %, 83.9 % and 78.6 %).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define FPG_BM_FN __host__ __device__ __forceinline__
#else
#define FPG_BM_FN inline
#endif

namespace fpg {

FPG_BM_FN uint32_t bm_bits(float x) {
    uint32_t b;
    std::memcpy(&b, &x, sizeof b);
    return b;
}

FPG_BM_FN float bm_float(uint32_t b) {
    float x;
    std::memcpy(&x, &b, sizeof x);
    return x;
}

// ln u for a normal u in (0, 1).
FPG_BM_FN float bm_log(float u) {
    const uint32_t b = bm_bits(u);
    const int32_t e = (int32_t)(b - 0x3f3504f3u) >> 23;       // 0x3f3504f3: the float just below 1/sqrt2
    const float m = bm_float(b - ((uint32_t)e << 23));        // u / 2^e in [1/sqrt2, sqrt2)
    const float f = m - 1.0f;
    const float f2 = f * f;
    float q = -0x1.383114p-4f;
    q = fmaf(q, f, 0x1.0848f6p-3f);
    q = fmaf(q, f, -0x1.0f377cp-3f);
    q = fmaf(q, f, 0x1.227186p-3f);
    q = fmaf(q, f, -0x1.542768p-3f);
    q = fmaf(q, f, 0x1.99a3f4p-3f);
    q = fmaf(q, f, -0x1.000426p-2f);
    q = fmaf(q, f, 0x1.555550p-2f);
    q = fmaf(q, f, -0x1.fffff8p-2f);
    const float r = fmaf(f2, q, f);
    const float fe = (float)e;
    return fmaf(fe, 0x1.62e400p-1f, fmaf(fe, 0x1.7f7d1cp-20f, r));   // ln2 = 0x1.62e4p-1 + 0x1.7f7d1cp-20
}

// sin and cos of theta in [0, 2pi).
FPG_BM_FN void bm_sincos(float theta, float* sin_out, float* cos_out) {
    const float qf = rintf(theta * 0x1.45f306p-1f);            // 2/pi
    const int q = (int)qf;
    // pi/2 = 0x1.921fb6p+0 - 0x1.777a5cp-25 - 0x1.ee59dap-50 (each part the
    // float nearest to what the parts before leave)
    const float r1 = fmaf(-qf, 0x1.921fb6p+0f, theta);
    const float r = fmaf(-qf, -0x1.ee59dap-50f, fmaf(-qf, -0x1.777a5cp-25f, r1));
    const float r2 = r * r;
    const float ps = fmaf(fmaf(-0x1.994068p-13f, r2, 0x1.110730p-7f), r2, -0x1.555546p-3f);
    const float sn = fmaf(r * r2, ps, r);
    const float pc = fmaf(fmaf(0x1.99e86ap-16f, r2, -0x1.6c0c28p-10f), r2, 0x1.55554ap-5f);
    const float cs = 1.0f - fmaf(r2, 0.5f, -(r2 * r2) * pc);
    float s = (q & 1) ? cs : sn, c = (q & 1) ? sn : cs;
    if (q & 2) s = -s;
    if ((q + 1) & 2) c = -c;
    *sin_out = s;
    *cos_out = c;
}

}  // namespace fpg
