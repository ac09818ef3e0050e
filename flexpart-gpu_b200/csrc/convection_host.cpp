// convection_host.cpp — the simplified Emanuel convection column and its
// redistribution matrix, built on the host as the reference builds them
// (physics/convection.rs:222-355; matrix generation stays on the CPU there
// too, src/gpu/convection.rs:6-7).  Single-precision arithmetic in the
// reference's operation order; the device applies the matrix
// (fpg_convection_set_matrix / fpg_convective_mixing in cbl.cu).
#include <cmath>
#include <vector>

#include "../../include/fpg.h"

namespace {

constexpr float kCapeFromWstar = 350.0f;
constexpr float kCapeFromPrecip = 35.0f;
constexpr float kCapeActivation = 5.0f;
constexpr float kPrecipActivation = 0.05f;
constexpr float kMinTimescale = 300.0f;
constexpr float kMaxTimescale = 3600.0f;
constexpr float kMassFluxScale = 0.02f;
constexpr float kDepthOffset = 1500.0f;
constexpr float kCapeDepthFactor = 20.0f;

float clampf_host(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }

}  // namespace

// level_index_from_height (physics/convection.rs:469-489).
extern "C" size_t fpg_convection_level_index(const float* iface, size_t n_interfaces, float height_m) {
    if (!iface || n_interfaces < 2) return 0;
    const size_t L = n_interfaces - 1;
    const float z = std::fmin(std::fmax(height_m, iface[0]), iface[L]);
    for (size_t l = 0; l < L; ++l)
        if (z >= iface[l] && z < iface[l + 1]) return l;
    return L - 1;
}

extern "C" fpg_status fpg_convection_build_chain(const fpg_convection_inputs* in, float dt_seconds,
                                                 fpg_convection_column* column, float* matrix_out,
                                                 float* centers_out, float* mass_flux_out,
                                                 float* detrainment_out) {
    if (!in || !column || !matrix_out) return FPG_ERR_INVALID_ARGUMENT;
    const float* iface = in->level_interfaces_m;
    const size_t n_if = in->n_interfaces;
    // SimplifiedEmanuelInputs::validate (physics/convection.rs:84-108)
    if (n_if < 2 || !iface) return FPG_ERR_TOO_FEW_LEVELS;
    for (size_t i = 0; i + 1 < n_if; ++i)
        if (!std::isfinite(iface[i]) || !std::isfinite(iface[i + 1]) || iface[i + 1] <= iface[i])
            return FPG_ERR_NON_MONOTONIC_INTERFACES;
    const float hbl = in->boundary_layer_height_m;
    if (!std::isfinite(hbl) || hbl < 0.0f) return FPG_ERR_INVALID_BOUNDARY_LAYER_HEIGHT;

    // compute_simplified_emanuel_column (physics/convection.rs:222-321)
    const size_t L = n_if - 1;
    std::vector<float> centers(L), flux(L, 0.0f), det(L, 0.0f);
    for (size_t l = 0; l < L; ++l) centers[l] = 0.5f * (iface[l] + iface[l + 1]);
    const float precip = in->convective_precip_mm_h;
    float cape;
    if (in->has_cape_override) {
        cape = in->cape_override_j_kg;
    } else {
        const float wstar = std::fmax(in->convective_velocity_scale_m_s, 0.0f);
        cape = kCapeFromWstar * wstar * wstar + kCapeFromPrecip * std::fmax(precip, 0.0f);
    }
    const bool active = cape >= kCapeActivation && precip >= kPrecipActivation;
    fpg_convection_column col{};
    size_t base = 0, top = 0;
    float timescale = kMaxTimescale;
    if (active) {
        const float column_top = iface[L];
        const float base_h = std::fmin(std::fmax(0.6f * hbl, iface[0]), column_top);
        base = fpg_convection_level_index(iface, n_if, base_h);
        const float depth = kDepthOffset + kCapeDepthFactor * std::sqrt(cape);
        const float top_h = std::fmin(std::fmax(base_h + depth, base_h), column_top);
        top = fpg_convection_level_index(iface, n_if, top_h);
        if (top < base) top = base;
        const size_t span = top - base;
        const float peak = kMassFluxScale * std::sqrt(cape) * (1.0f + 0.1f * std::fmax(precip, 0.0f));
        float sum = 0.0f;
        for (size_t l = base; l <= top; ++l) {
            const float normalized = span == 0 ? 0.5f : (float)(l - base) / (float)span;
            const float bell = std::fmax(4.0f * normalized * (1.0f - normalized), 0.0f);
            const float f = peak * (0.05f + bell);
            flux[l] = f;
            det[l] = f;
            sum += f;
        }
        if (sum > 0.0f) {
            for (size_t l = 0; l < L; ++l) det[l] /= sum;
        } else {
            const size_t count = top - base + 1;
            for (size_t l = base; l <= top; ++l) det[l] = 1.0f / (float)count;
        }
        const float intensity = clampf_host(cape / 1200.0f + std::fmax(precip, 0.0f) / 20.0f, 0.0f, 1.0f);
        timescale = kMaxTimescale - intensity * (kMaxTimescale - kMinTimescale);
    }
    col.is_active = active ? 1 : 0;
    col.cape_j_kg = active ? cape : std::fmax(cape, 0.0f);
    col.cloud_base_level = (uint32_t)base;
    col.cloud_top_level = (uint32_t)top;
    col.convective_timescale_s = timescale;
    col.mixing_fraction = 0.0f;

    // build_convective_redistribution_matrix (physics/convection.rs:324-367)
    if (!std::isfinite(dt_seconds) || dt_seconds <= 0.0f) return FPG_ERR_INVALID_TIME_STEP;
    for (size_t i = 0; i < L * L; ++i) matrix_out[i] = 0.0f;
    for (size_t l = 0; l < L; ++l) matrix_out[l * L + l] = 1.0f;
    if (active) {
        const float ts = clampf_host(timescale, kMinTimescale, kMaxTimescale);
        const float cape_factor = clampf_host(cape / (cape + 100.0f), 0.0f, 1.0f);
        const float mixing = clampf_host((1.0f - std::exp(-dt_seconds / ts)) * cape_factor, 0.0f, 0.95f);
        for (size_t s = base; s <= top; ++s) {
            for (size_t d = 0; d < L; ++d) {
                float v = mixing * det[d];
                if (d == s) v += 1.0f - mixing;
                matrix_out[s * L + d] = v;
            }
        }
        col.mixing_fraction = mixing;
        // ConvectiveRedistributionMatrix::from_column_major validation
        for (size_t s = 0; s < L; ++s) {
            float sum = 0.0f;
            for (size_t d = 0; d < L; ++d) {
                const float w = matrix_out[s * L + d];
                if (w < -1.0e-4f || !std::isfinite(w)) return FPG_ERR_NON_STOCHASTIC_COLUMN;
                sum += w;
            }
            if (std::fabs(sum - 1.0f) > 1.0e-4f) return FPG_ERR_NON_STOCHASTIC_COLUMN;
        }
    }
    *column = col;
    for (size_t l = 0; l < L; ++l) {
        if (centers_out) centers_out[l] = centers[l];
        if (mass_flux_out) mass_flux_out[l] = flux[l];
        if (detrainment_out) detrainment_out[l] = det[l];
    }
    return FPG_OK;
}

// apply_redistribution_matrix (physics/convection.rs:370-392): destination =
// M * source, accumulated source level by source level.
extern "C" fpg_status fpg_convection_apply_profile(const float* matrix_column_major, size_t level_count,
                                                   const float* source, size_t n_source, float* destination) {
    if (!matrix_column_major || !source || !destination) return FPG_ERR_INVALID_ARGUMENT;
    if (n_source != level_count) return FPG_ERR_LENGTH_MISMATCH;
    const size_t L = level_count;
    for (size_t d = 0; d < L; ++d) destination[d] = 0.0f;
    for (size_t s = 0; s < L; ++s)
        for (size_t d = 0; d < L; ++d) destination[d] += matrix_column_major[s * L + d] * source[s];
    return FPG_OK;
}
