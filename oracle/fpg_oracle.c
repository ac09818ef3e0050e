/*
 * fpg_oracle.c — parity oracle for the flexpart-gpu per-particle step.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
 * oracle/_build/liborc.so.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it; the CUDA library (libfpg) never
 * links it and has no CPU fallback.
 *
 * Integer parts (Philox, counters, release bookkeeping, compaction order) are
 * written once; floating-point physics lives in oracle_core.inc, compiled for
 * float (the parity build, *_f32) and for double (the FP64 error reference,
 * *_f64).  Pinning: tests/test_oracle_golden.py checks this file against every
 * known-answer vector and analytic test of the reference that covers the
 * path (Philox KAT and carry, Langevin zero-noise update, trilinear corner /
 * centre / linear / clamp cases, advection analytic uniform and shear flows,
 * Hanna table ratios and no-NaN sweep, gridding parity case, deposition
 * decay, alpha sequence, release counts and bounds, compaction sets).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/fpg.h"

/* ---- Philox4x32-10 (src/physics/rng.rs:14-96) --------------------------- */

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

/* philox_round + raise_key, 10 rounds (rng.rs:28-65). */
void orc_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = counter[0], c1 = counter[1], c2 = counter[2], c3 = counter[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* philox_counter_add (rng.rs:69-87): 128-bit add of a 64-bit offset. */
void orc_counter_add_u64(const uint32_t counter[4], uint64_t offset, uint32_t out[4]) {
    uint32_t low = (uint32_t)offset, high = (uint32_t)(offset >> 32);
    uint32_t c0 = counter[0] + low;
    uint32_t carry0 = c0 < counter[0];
    uint32_t n1 = counter[1] + high;
    uint32_t carry1a = n1 < counter[1];
    uint32_t c1 = n1 + carry0;
    uint32_t carry1b = c1 < n1;
    uint32_t carry1 = carry1a | carry1b;
    uint32_t c2 = counter[2] + carry1;
    uint32_t carry2 = c2 < counter[2];
    uint32_t c3 = counter[3] + carry2;
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* counter_add with a u32 offset, as the shader does it
 * (langevin_fused.wgsl:171-180). */
void orc_counter_add_u32(const uint32_t base[4], uint32_t offset, uint32_t out[4]) {
    uint32_t c0 = base[0] + offset;
    uint32_t carry0 = c0 < base[0];
    uint32_t c1 = base[1] + carry0;
    uint32_t carry1 = (carry0 == 1u) && (c1 < base[1]);
    uint32_t c2 = base[2] + carry1;
    uint32_t carry2 = (carry1 == 1u) && (c2 < base[2]);
    uint32_t c3 = base[3] + carry2;
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* u32_to_uniform01 (rng.rs:94-96): high 24 bits times 2^-24. */
float orc_u32_to_uniform01(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

/* philox4x32_uniforms over n consecutive blocks (rng.rs:100-108); raw may be NULL. */
void orc_philox_uniforms(const uint32_t key[2], const uint32_t counter[4], size_t n_blocks,
                         float* out, uint32_t* raw) {
    for (size_t b = 0; b < n_blocks; ++b) {
        uint32_t c[4], blk[4];
        orc_counter_add_u64(counter, (uint64_t)b, c);
        orc_philox4x32_10(c, key, blk);
        for (int k = 0; k < 4; ++k) {
            if (out) out[4 * b + k] = orc_u32_to_uniform01(blk[k]);
            if (raw) raw[4 * b + k] = blk[k];
        }
    }
}

/* Host-side counter advance of one fused Langevin dispatch
 * (gpu/langevin_fused.rs:229-233). */
void orc_next_counter(const uint32_t base[4], uint64_t particle_count, uint32_t n_substeps,
                      uint32_t out[4]) {
    if (particle_count == 0) { memcpy(out, base, 16); return; }
    uint64_t blocks_per_particle = n_substeps <= 2u ? 1u : 2u;
    orc_counter_add_u64(base, particle_count * blocks_per_particle, out);
}

/* ---- FP32 and FP64 physics ---------------------------------------------- */

#define R float
#define SFX _f32
#define FMA fmaf
#define FMAX fmaxf
#define FMIN fminf
#define FABS fabsf
#define FLOOR floorf
#define SQRT sqrtf
#define EXP expf
#define LOG logf
#define POW powf
#define SIN sinf
#define COS cosf
#define ONE_THIRD (1.0f / 3.0f)
#define TWO_THIRDS (2.0f / 3.0f)
#define TWO_PI_R 6.2831855f
#include "oracle_core.inc"
#undef R
#undef SFX
#undef FMA
#undef FMAX
#undef FMIN
#undef FABS
#undef FLOOR
#undef SQRT
#undef EXP
#undef LOG
#undef POW
#undef SIN
#undef COS
#undef ONE_THIRD
#undef TWO_THIRDS
#undef TWO_PI_R

#define R double
#define SFX _f64
#define FMA fma
#define FMAX fmax
#define FMIN fmin
#define FABS fabs
#define FLOOR floor
#define SQRT sqrt
#define EXP exp
#define LOG log
#define POW pow
#define SIN sin
#define COS cos
#define ONE_THIRD (1.0 / 3.0)
#define TWO_THIRDS (2.0 / 3.0)
#define TWO_PI_R 6.283185307179586
#include "oracle_core.inc"

/* ---- Compaction order (compaction.wgsl:65-217) --------------------------- */

/* Stable scan of the active bit: out_indices[k] is the k-th active slot in
 * slot order (passes 1-3); returns the active count. */
uint32_t orc_compaction_indices(const uint32_t* flags, size_t n, uint32_t* out_indices) {
    uint32_t count = 0;
    for (size_t i = 0; i < n; ++i)
        if (flags[i] & 1u) out_indices[count++] = (uint32_t)i;
    return count;
}

/* Pass 4 (gather_reorder, compaction.wgsl:194-217) applied to one 4-byte
 * field: dst[g] = src[idx[g]] for g < active, else src[g]. */
void orc_compaction_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t active, size_t n,
                               uint32_t* dst) {
    for (size_t g = 0; g < n; ++g) dst[g] = g < active ? src[idx[g]] : src[g];
}

/* ---- Time bookkeeping (simulation/timeloop.rs:2086-2120; release/mod.rs) */

/* interpolation_alpha: f64 ratio cast to f32.  Returns FPG_ERR_INVALID_BRACKET
 * when t1 <= t0, FPG_ERR_OUTSIDE_BRACKET for an outside target in strict mode. */
int32_t orc_interpolation_alpha(int64_t t0, int64_t t1, int64_t target, int32_t clamp_mode,
                                float* out) {
    if (t1 <= t0) return FPG_ERR_INVALID_BRACKET;
    int64_t eff = target;
    if (!(target >= t0 && target <= t1)) {
        if (!clamp_mode) return FPG_ERR_OUTSIDE_BRACKET;
        eff = target < t0 ? t0 : t1;
    }
    double elapsed = (double)(eff - t0);
    double window = (double)(t1 - t0);
    *out = (float)(elapsed / window);
    return FPG_OK;
}

/* days_from_civil (release/mod.rs:337-351). */
static int64_t days_from_civil(int64_t y, int64_t m, int64_t d) {
    if (m <= 2) y -= 1;
    int64_t era = (y >= 0 ? y : y - 399) / 400;
    int64_t yoe = y - era * 400;
    int64_t mp = m + (m > 2 ? -3 : 9);
    int64_t doy = (153 * mp + 2) / 5 + d - 1;
    int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + doe - 719468;
}

/* parse_timestamp_seconds (release/mod.rs:283-334): "YYYYMMDDHHMMSS". */
int32_t orc_parse_timestamp(const char* s, int64_t* out) {
    if (strlen(s) != 14) return FPG_ERR_INVALID_ARGUMENT;
    int v[14];
    for (int i = 0; i < 14; ++i) {
        if (s[i] < '0' || s[i] > '9') return FPG_ERR_INVALID_ARGUMENT;
        v[i] = s[i] - '0';
    }
    int64_t year = v[0] * 1000 + v[1] * 100 + v[2] * 10 + v[3];
    int64_t month = v[4] * 10 + v[5], day = v[6] * 10 + v[7];
    int64_t hour = v[8] * 10 + v[9], minute = v[10] * 10 + v[11], second = v[12] * 10 + v[13];
    if (month < 1 || month > 12 || day < 1 || day > 31 || hour > 23 || minute > 59 || second > 59)
        return FPG_ERR_INVALID_ARGUMENT;
    *out = days_from_civil(year, month, day) * 86400 + hour * 3600 + minute * 60 + second;
    return FPG_OK;
}

/* ReleaseState::target_emitted_count (release/mod.rs:181-196). */
uint64_t orc_target_emitted_count(uint64_t particle_count, int64_t start, int64_t end, int64_t now,
                                  uint64_t released_count) {
    if (now < start || now > end) return released_count;
    if (start == end) return particle_count;
    if (now == end) return particle_count;
    unsigned __int128 e = (unsigned __int128)(uint64_t)(now - start);
    unsigned __int128 d = (unsigned __int128)(uint64_t)(end - start);
    return (uint64_t)(((unsigned __int128)particle_count * e) / d);
}

/* ReleaseBounds::sample_stratified (release/mod.rs:256-275).
 * bounds: lon_min, lon_max, lat_min, lat_max, z_min, z_max. */
void orc_sample_stratified(const double bounds[6], uint64_t sample_index, uint64_t total,
                           double out[3]) {
    double c = ceil(cbrt((double)total));
    if (c < 1.0) c = 1.0;
    uint64_t nx = (uint64_t)c;
    uint64_t ny = nx;
    uint64_t nxy = nx * ny;
    if (nxy < 1) nxy = 1;
    uint64_t nz = (total + nxy - 1) / nxy;
    if (nz < 1) nz = 1;
    uint64_t ix = sample_index % nx;
    uint64_t iy = (sample_index / nx) % ny;
    uint64_t iz = (sample_index / nxy) % nz;
    double fx = ((double)ix + 0.5) / (double)nx;
    double fy = ((double)iy + 0.5) / (double)ny;
    double fz = ((double)iz + 0.5) / (double)nz;
    out[0] = bounds[0] + fx * (bounds[1] - bounds[0]);
    out[1] = bounds[2] + fy * (bounds[3] - bounds[2]);
    out[2] = bounds[4] + fz * (bounds[5] - bounds[4]);
}

/* geo_to_grid + GridDomain::contains + GridCoord::to_relative
 * (coords/mod.rs:92-94,109-114,169-178).  domain: xlon0, ylat0, dx, dy, nx, ny. */
int32_t orc_geo_to_relative(double lon, double lat, const double domain[6], int32_t* cell_x,
                            int32_t* cell_y, float* frac_x, float* frac_y) {
    double x = (lon - domain[0]) / domain[2];
    double y = (lat - domain[1]) / domain[3];
    double nx = domain[4], ny = domain[5];
    if (!(x >= 0.0 && x < nx - 1.0 && y >= 0.0 && y < ny - 1.0)) return FPG_ERR_OUT_OF_GRID;
    double fx = floor(x), fy = floor(y);
    *cell_x = (int32_t)fx;
    *cell_y = (int32_t)fy;
    *frac_x = (float)(x - fx);
    *frac_y = (float)(y - fy);
    return FPG_OK;
}

/* wet_precipitation_state + below_cloud_scavenging_coefficient_gas
 * (physics/wet_scavenging.rs:179-225,405-430) for one cell: returns lambda
 * [1/s] and precipitating fraction. */
static float snn0(float v) { return (isfinite(v) && v > 0.0f) ? v : 0.0f; }
static int precip_class(float p) {
    if (p > 20.0f) return 4;
    if (p > 8.0f) return 3;
    if (p > 3.0f) return 2;
    if (p > 1.0f) return 1;
    return 0;
}
void orc_wet_cell(float lsp_in, float convp_in, float cloud_cover, float a_in, float b_in,
                  float* lambda_out, float* fraction_out) {
    static const float lsf[5] = {0.5f, 0.65f, 0.8f, 0.9f, 0.95f};
    static const float cvf[5] = {0.4f, 0.55f, 0.7f, 0.8f, 0.9f};
    float lsp = snn0(lsp_in), convp = snn0(convp_in);
    float total = lsp + convp;
    float fraction = 0.0f, subgrid = 0.0f;
    if (!(total < 0.01f)) {
        float cc = fminf(fmaxf(cloud_cover, 0.0f), 1.0f);
        float weighted = (lsp * lsf[precip_class(lsp)] + convp * cvf[precip_class(convp)]) /
                         fmaxf(total, 1.0e-12f);
        float area = fminf(fmaxf(fmaxf(cc * weighted, 0.05f), 0.05f), 1.0f);
        subgrid = snn0(total / fmaxf(area, 1.0e-12f));
        fraction = area;
    }
    /* WetPrecipitationState::is_active (wet_scavenging.rs:78-82) gates the
     * coefficient; an inactive cell scavenges nothing. */
    float lambda = 0.0f;
    int active = total >= 0.01f && fraction > 0.0f && subgrid > 0.0f;
    if (active) {
        float a = snn0(a_in), b = snn0(b_in);
        lambda = snn0(a * powf(subgrid, b));
    } else {
        fraction = 0.0f;
    }
    *lambda_out = lambda;
    *fraction_out = fraction;
}

/* orc_wet_cell over a grid of n cells (convp / cloud_cover may be NULL:
 * 0 and 1). */
void orc_wet_cells_grid(size_t n, const float* lsp, const float* convp, const float* cloud_cover, float a,
                        float b, float* lambda_out, float* fraction_out) {
    for (size_t c = 0; c < n; ++c)
        orc_wet_cell(lsp[c], convp ? convp[c] : 0.0f, cloud_cover ? cloud_cover[c] : 1.0f, a, b, &lambda_out[c],
                     &fraction_out[c]);
}

/* interpolate_wind_field_linear's per-value lerp (io/temporal.rs:67-120,
 * 417-420: a.mul_add(1 - t, b * t)) over n values, as the reference's CPU
 * pipeline time-interpolates a whole wind component before advecting
 * (benches/advection.rs:1138-1146). */
void orc_lerp_field(size_t n, const float* a, const float* b, float t, float* out, int n_threads) {
    const float s = 1.0f - t;
#pragma omp parallel for schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (long long i = 0; i < (long long)n; ++i) out[i] = fmaf(a[i], s, b[i] * t);
}

/* ---- CBL skewed vertical-velocity PDF (physics/cbl.rs) ------------------
 * pdf[11] = updraft weight, mean, sigma; downdraft weight, mean, sigma;
 * target w2, w3, skewness; transition; z/h.  f32 throughout, as the CPU
 * routines run: cbrtf for f32::cbrt, powf for powf, repeated products for
 * powi. */

/* cbl_transition_factor (physics/cbl.rs:109-124). */
float orc_cbl_transition_factor(float h, float ol) {
    if (!isfinite(h) || h <= 0.0f || !isfinite(ol) || ol == 0.0f) return 1.0f;
    float ratio = -h / ol;
    float t = ratio < 15.0f ? sinf(((ratio + 10.0f) / 10.0f) * 3.14159265358979323846f) * 0.5f + 0.5f : 1.0f;
    return fminf(fmaxf(t, 0.0f), 1.0f);
}

/* compute_cbl_moments + compute_cbl_bigaussian_pdf (physics/cbl.rs:126-226);
 * in[5] = z, h, w*, sigma_w, L. */
void orc_cbl_pdf(const float in[5], float pdf[11]) {
    float h = fmaxf(in[1], 1.0f);
    float z = fminf(fmaxf(in[0], 0.0f), h);
    float zoh = z / h;
    float wst = fmaxf(in[2], 0.0f);
    float sw = fmaxf(in[3], 1.0e-5f);
    float trans = orc_cbl_transition_factor(h, in[4]);
    float w2 = sw * sw;
    float shape = 1.2f * zoh * powf(1.0f - zoh, 1.5f) + 1.0e-6f;
    float w3 = shape * (wst * wst * wst) * trans;
    float skew = w3 / powf(w2, 1.5f);
    float sym[11] = {0.5f, 0.0f, sw, 0.5f, 0.0f, sw, w2, w3, skew, trans, zoh};
    memcpy(pdf, sym, sizeof(sym));
    if (!isfinite(skew) || fabsf(skew) <= 1.0e-6f) return;
    float fl = (2.0f / 3.0f) * cbrtf(skew);
    float fl2 = fl * fl;
    if (!isfinite(fl) || fabsf(fl) <= 1.0e-6f) return;
    float skew2 = skew * skew;
    float a1 = 1.0f + fl2, a3 = 3.0f + fl2;
    float num = (a1 * a1 * a1) * skew2;
    float den = (a3 * a3) * fl2;
    float r = fmaxf(num / fmaxf(den, 1.0e-6f), 0.0f);
    float x = sqrtf(r);
    float aw = 0.5f * (1.0f - x / sqrtf(4.0f + r));
    aw = fminf(fmaxf(aw, 1.0e-4f), 1.0f - 1.0e-4f);
    float bw = 1.0f - aw;
    float sa = sw * sqrtf(bw / (aw * (1.0f + fl2)));
    float sb = sw * sqrtf(aw / (bw * (1.0f + fl2)));
    pdf[0] = aw; pdf[1] = fl * sa; pdf[2] = fmaxf(sa, 1.0e-5f);
    pdf[3] = bw; pdf[4] = -(fl * sb); pdf[5] = fmaxf(sb, 1.0e-5f);
}

/* reconstruct_cbl_moments (physics/cbl.rs:229-255): out = w2, w3, skewness. */
void orc_cbl_reconstruct_moments(const float pdf[11], float out[3]) {
    float wa = pdf[0], wb = pdf[3], ma = pdf[1], mb = pdf[4];
    float s2a = pdf[2] * pdf[2], s2b = pdf[5] * pdf[5];
    float w2 = wa * (s2a + ma * ma) + wb * (s2b + mb * mb);
    float w3 = wa * ((ma * ma * ma) + 3.0f * ma * s2a) + wb * ((mb * mb * mb) + 3.0f * mb * s2b);
    out[0] = w2;
    out[1] = w3;
    out[2] = w2 > 0.0f ? w3 / powf(w2, 1.5f) : 0.0f;
}

static float cbl_normal_pdf(float v, float mean, float sigma) {
    sigma = fmaxf(sigma, 1.0e-5f);
    float s = (v - mean) / sigma;
    return (0.3989423f / sigma) * expf(-0.5f * s * s);
}

/* CblBiGaussianPdf::probability_density (physics/cbl.rs:257-270). */
float orc_cbl_probability_density(const float pdf[11], float w) {
    return pdf[0] * cbl_normal_pdf(w, pdf[1], pdf[2]) + pdf[3] * cbl_normal_pdf(w, pdf[4], pdf[5]);
}

/* sample_cbl_vertical_velocity (physics/cbl.rs:274-288). */
float orc_cbl_sample(const float pdf[11], float ub, float u0, float u1) {
    float bm[2];
    orc_box_muller_f32(u0, u1, bm);
    return ub < pdf[0] ? pdf[1] + pdf[2] * bm[0] : pdf[4] + pdf[5] * bm[0];
}

/* sample_cbl_vertical_velocity_with_rng (physics/cbl.rs:291-295): each call
 * takes the four uniforms of one Philox block (next_uniform4 on a stream
 * whose cache is empty, physics/rng.rs:130-164) and advances the counter. */
float orc_cbl_sample_with_rng(const float pdf[11], const uint32_t key[2], uint32_t counter[4]) {
    uint32_t b[4], next[4];
    orc_philox4x32_10(counter, key, b);
    orc_counter_add_u32(counter, 1u, next);
    memcpy(counter, next, 16);
    return orc_cbl_sample(pdf, orc_u32_to_uniform01(b[0]), orc_u32_to_uniform01(b[1]), orc_u32_to_uniform01(b[2]));
}

/* infer_cbl_branch (physics/cbl.rs:300-309): 1 updraft, 0 downdraft. */
int32_t orc_cbl_infer_branch(float previous_w, int32_t time_direction) {
    float sign = previous_w > 0.0f ? 1.0f : (previous_w < 0.0f ? -1.0f : (signbit(previous_w) ? -1.0f : 1.0f));
    if (isnan(previous_w)) sign = previous_w;
    float signed_w = sign * (time_direction >= 0 ? 1.0f : -1.0f);
    return signed_w >= 0.0f ? 1 : 0;
}

/* sample_cbl_branch_constrained_velocity (physics/cbl.rs:315-331). */
float orc_cbl_branch_constrained(const float pdf[11], int32_t updraft, float u0, float u1, int32_t time_direction) {
    float bm[2];
    orc_box_muller_f32(u0, u1, bm);
    float eta = bm[0];
    float speed = updraft ? fabsf(pdf[1] + pdf[2] * eta) : -(fabsf(pdf[4]) + pdf[5] * fabsf(eta));
    return speed * (time_direction >= 0 ? 1.0f : -1.0f);
}

/* The dispatch of src/gpu/cbl.rs (cbl.wgsl:251-298) over n slots: hanna16 is
 * HannaParams records (h at [3], w* at [1], L at [2], sigma_w at [7]), in4
 * the sampling inputs; out12 = sample, pdf[11]; zeros for inactive slots. */
void orc_cbl_sample_slots(size_t n, const uint32_t* flags, const float* pos_z, const float* hanna16,
                          const float* in4, float* out12) {
    for (size_t p = 0; p < n; ++p) {
        float* o = out12 + 12 * p;
        if (!(flags[p] & 1u)) { memset(o, 0, 12 * sizeof(float)); continue; }
        const float* hp = hanna16 + 16 * p;
        float in[5] = {pos_z[p], hp[3], hp[1], hp[7], hp[2]};
        float pdf[11];
        orc_cbl_pdf(in, pdf);
        o[0] = orc_cbl_sample(pdf, in4[4 * p], in4[4 * p + 1], in4[4 * p + 2]);
        memcpy(o + 1, pdf, sizeof(pdf));
    }
}

/* compute_hanna_params_gpu (hanna_params.wgsl:231-258) over n slots with
 * compute_hanna_params_from_pbl (physics/hanna.rs:178-194); out16 records,
 * zeros for inactive slots. */
void orc_hanna_params_slots(size_t n, const int32_t* cell_x, const int32_t* cell_y, const float* pos_x,
                            const float* pos_y, const float* pos_z, const uint32_t* flags, const float* ustar,
                            const float* wstar, const float* hmix, const float* oli, size_t pnx, size_t pny,
                            float* out16) {
    for (size_t p = 0; p < n; ++p) {
        float* o = out16 + 16 * p;
        memset(o, 0, 16 * sizeof(float));
        if (!(flags[p] & 1u)) continue;
        float x = (float)cell_x[p] + pos_x[p];
        float y = (float)cell_y[p] + pos_y[p];
        size_t i = (size_t)floorf(fminf(fmaxf(x, 0.0f), (float)(pnx - 1)));
        size_t j = (size_t)floorf(fminf(fmaxf(y, 0.0f), (float)(pny - 1)));
        size_t c = i * pny + j;
        orc_hanna_f32(ustar[c], wstar[c], orc_obukhov_from_inverse_f32(oli[c]), hmix[c], pos_z[p], o);
    }
}

/* ---- Convection chain (physics/convection.rs) --------------------------- */

/* level_index_from_height (physics/convection.rs:469-489). */
size_t orc_level_index_from_height(const float* iface, size_t n_iface, float height) {
    size_t L = n_iface > 0 ? n_iface - 1 : 0;
    if (L == 0) return 0;
    float z = fminf(fmaxf(height, iface[0]), iface[L]);
    for (size_t l = 0; l < L; ++l)
        if (z >= iface[l] && z < iface[l + 1]) return l;
    return L - 1;
}

/* build_simplified_convection_chain (physics/convection.rs:222-367, 462-467).
 * info[6] = is_active, cape, cloud base, cloud top, timescale, mixing
 * fraction.  Returns 0 or the FPG_ERR_* of the reference error. */
int32_t orc_convection_chain(const float* iface, size_t n_iface, float precip, float wstar_in, float hbl,
                             int32_t has_cape, float cape_override, float dt, float* matrix, float* det_out,
                             float* info) {
    if (n_iface < 2) return FPG_ERR_TOO_FEW_LEVELS;
    for (size_t i = 0; i + 1 < n_iface; ++i)
        if (!isfinite(iface[i]) || !isfinite(iface[i + 1]) || iface[i + 1] <= iface[i])
            return FPG_ERR_NON_MONOTONIC_INTERFACES;
    if (!isfinite(hbl) || hbl < 0.0f) return FPG_ERR_INVALID_BOUNDARY_LAYER_HEIGHT;
    size_t L = n_iface - 1;
    float cape;
    if (has_cape) {
        cape = cape_override;
    } else {
        float w = fmaxf(wstar_in, 0.0f);
        cape = 350.0f * w * w + 35.0f * fmaxf(precip, 0.0f);
    }
    int active = cape >= 5.0f && precip >= 0.05f;
    float* det = calloc(L, sizeof(float));
    size_t base = 0, top = 0;
    float timescale = 3600.0f;
    if (active) {
        float ctop = iface[L];
        float base_h = fminf(fmaxf(0.6f * hbl, iface[0]), ctop);
        base = orc_level_index_from_height(iface, n_iface, base_h);
        float depth = 1500.0f + 20.0f * sqrtf(cape);
        float top_h = fminf(fmaxf(base_h + depth, base_h), ctop);
        top = orc_level_index_from_height(iface, n_iface, top_h);
        if (top < base) top = base;
        size_t span = top - base;
        float peak = 0.02f * sqrtf(cape) * (1.0f + 0.1f * fmaxf(precip, 0.0f));
        float sum = 0.0f;
        for (size_t l = base; l <= top; ++l) {
            float nrm = span == 0 ? 0.5f : (float)(l - base) / (float)span;
            float bell = fmaxf(4.0f * nrm * (1.0f - nrm), 0.0f);
            float f = peak * (0.05f + bell);
            det[l] = f;
            sum += f;
        }
        if (sum > 0.0f) {
            for (size_t l = 0; l < L; ++l) det[l] /= sum;
        } else {
            for (size_t l = base; l <= top; ++l) det[l] = 1.0f / (float)(top - base + 1);
        }
        float intensity = fminf(fmaxf(cape / 1200.0f + fmaxf(precip, 0.0f) / 20.0f, 0.0f), 1.0f);
        timescale = 3600.0f - intensity * (3600.0f - 300.0f);
    }
    if (!isfinite(dt) || dt <= 0.0f) { free(det); return FPG_ERR_INVALID_TIME_STEP; }
    memset(matrix, 0, L * L * sizeof(float));
    for (size_t l = 0; l < L; ++l) matrix[l * L + l] = 1.0f;
    float mixing = 0.0f;
    if (active) {
        float ts = fminf(fmaxf(timescale, 300.0f), 3600.0f);
        float cf = fminf(fmaxf(cape / (cape + 100.0f), 0.0f), 1.0f);
        mixing = fminf(fmaxf((1.0f - expf(-dt / ts)) * cf, 0.0f), 0.95f);
        for (size_t s = base; s <= top; ++s)
            for (size_t d = 0; d < L; ++d) {
                float v = mixing * det[d];
                if (d == s) v += 1.0f - mixing;
                matrix[s * L + d] = v;
            }
    }
    if (det_out) memcpy(det_out, det, L * sizeof(float));
    free(det);
    info[0] = (float)active;
    info[1] = active ? cape : fmaxf(cape, 0.0f);
    info[2] = (float)base;
    info[3] = (float)top;
    info[4] = timescale;
    info[5] = mixing;
    return FPG_OK;
}

/* apply_convective_mixing_to_particles_cpu (physics/convection.rs:431-459)
 * with expected_destination_height_m (physics/convection.rs:398-427). */
void orc_convective_mixing(size_t n, const uint32_t* flags, float* pos_z, int32_t* cbt, const float* matrix,
                           size_t L, const float* iface, const float* centers) {
    float zmin = iface[0], zmax = iface[L];
    for (size_t p = 0; p < n; ++p) {
        if (!(flags[p] & 1u)) continue;
        size_t s = orc_level_index_from_height(iface, L + 1, pos_z[p]);
        float wh = 0.0f, sum = 0.0f;
        for (size_t d = 0; d < L; ++d) {
            float w = fmaxf(matrix[s * L + d], 0.0f);
            wh += w * centers[d];
            sum += w;
        }
        float dest = sum > 0.0f ? wh / sum : centers[s];
        pos_z[p] = fminf(fmaxf(dest, zmin), zmax);
        cbt[p] = (int32_t)s;
    }
}

/* n successive sample_cbl_vertical_velocity_with_rng calls on one stream. */
void orc_cbl_sample_stream(const float pdf[11], const uint32_t key[2], const uint32_t counter[4], size_t n,
                           float* out) {
    uint32_t c[4];
    memcpy(c, counter, 16);
    for (size_t i = 0; i < n; ++i) out[i] = orc_cbl_sample_with_rng(pdf, key, c);
}
