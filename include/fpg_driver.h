/*
 * fpg_driver.h — the forward time loop over the fpg.h kernels, the
 * replacement of the reference's ForwardTimeLoopDriver
 * (src/simulation/timeloop.rs:660-1431) for callers that want the whole
 * orchestration behind the C ABI rather than the individual seam functions.
 *
 * Per run_timestep, in the reference's order (timeloop.rs:915-1316):
 *   optional spatial reorder            (apply_spatial_sort_if_enabled, :1414-1430)
 *   release of the step's particles     (ReleaseManager::inject_and_upload_for_time,
 *                                        release/mod.rs:90-168)
 *   interpolation alpha                 (interpolation_alpha, :2086-2120)
 *   met bracket upload if it changed    (upload_dual_wind_if_bracket_changed, :1378-1402)
 *   surface lerp + PBL diagnostics      (io/temporal.rs:122, gpu/pbl.rs:367)
 *   fused advection + Langevin + dry + wet (fpg_step)
 *   optional compaction                 (encode_compaction_with_reorder, :1185-1262)
 * and the Philox counter advances by dispatch_count * blocks, as
 * encode_langevin_fused_gpu returns it (gpu/langevin_fused.rs:229-233).
 */
#ifndef FPG_DRIVER_H
#define FPG_DRIVER_H

#include "fpg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One release: ReleaseConfig as ReleaseManager reads it (release/mod.rs:199-254). */
typedef struct fpg_release {
    int64_t start_seconds;       /* seconds since 1970-01-01 (fpg_parse_timestamp) */
    int64_t end_seconds;
    double lon_min, lon_max;
    double lat_min, lat_max;
    double z_min, z_max;         /* metres above ground */
    double mass_kg;
    uint64_t particle_count;
} fpg_release;

/* GridDomain (src/coords/mod.rs): lon/lat of the lower-left node, spacing, size. */
typedef struct fpg_grid_domain {
    double xlon0, ylat0, dx, dy;
    uint64_t nx, ny;
} fpg_grid_domain;

/* ForwardTimeLoopConfig (timeloop.rs:67-124). */
typedef struct fpg_forward_config {
    int64_t start_seconds, end_seconds;   /* inclusive */
    int64_t timestep_seconds;
    int32_t clamp_time_bounds;            /* TimeBoundsBehavior: 1 Clamp, 0 Strict */
    float x_grid_per_meter, y_grid_per_meter, z_grid_per_meter;
    fpg_pbl_options pbl_options;
    float dry_reference_height_m;         /* 15 m */
    uint32_t philox_key[2];
    uint32_t initial_philox_counter[4];
    uint32_t sort_interval_steps;         /* 0: no spatial reorder */
    int32_t use_compaction;               /* FLEXPART_GPU_COMPACTION (timeloop.rs:506-513) */
    uint32_t n_substeps;                  /* 4 in production (timeloop.rs:1111) */
    float min_height_m;                   /* 0.01 in production (timeloop.rs:1112) */
} fpg_forward_config;

/* Fills the reference's defaults (timeloop.rs:107-124 and the production
 * Langevin step, :1108-1113). */
void fpg_forward_config_default(fpg_forward_config* cfg);

/* MetTimeBracket (timeloop.rs:270-285): host arrays, uploaded only when
 * (time_t0, time_t1) differs from the bracket already on the device. */
typedef struct fpg_met_bracket {
    const float *wind_t0_u, *wind_t0_v, *wind_t0_w;   /* nx*ny*nz, ((ix*ny)+iy)*nz+iz */
    const float *wind_t1_u, *wind_t1_v, *wind_t1_w;
    const fpg_surface_cell* surface_t0;              /* nx*ny, i*ny+j */
    const fpg_surface_cell* surface_t1;
    int64_t time_t0_seconds, time_t1_seconds;
} fpg_met_bracket;

/* ForwardStepForcing (timeloop.rs:347-358).  A mode of FPG_FORCING_NONE (or
 * UNIFORM with value 0) skips the process, as is_zero() does (:339-344).
 * PER_PARTICLE arrays are host arrays of `capacity` floats, uploaded every
 * step; PER_CELL uses `wet_cells` at the particle's nearest met cell. */
typedef struct fpg_forcing {
    int32_t dry_mode;
    float dry_velocity_m_s;
    const float* dry_velocity_per_slot;
    int32_t wet_mode;
    float wet_lambda_s_inv, wet_fraction;
    const float* wet_lambda_per_slot;
    const float* wet_fraction_per_slot;
    const fpg_cellfield* wet_cells;
    float rho_grad_over_rho;
} fpg_forcing;

/* ForwardStepReport (timeloop.rs:1294-1308). */
typedef struct fpg_step_report {
    uint64_t step_index;
    int64_t simulation_time_seconds;
    float interpolation_alpha;
    uint64_t released_count;
    uint64_t first_released_slot;
    uint64_t active_particle_count;
    uint32_t next_philox_counter[4];
} fpg_step_report;

typedef struct fpg_forward fpg_forward;

/* ForwardTimeLoopDriver::new (timeloop.rs:719-828): validates the config,
 * builds the release manager, allocates `capacity` particle slots and the
 * met, PBL and surface buffers of an nx*ny*nz met grid with the given level
 * heights (nz floats, or NULL for the level-index mode).  The particle
 * handle is owned by the driver (fpg_forward_particles). */
fpg_status fpg_forward_create(fpg_ctx* ctx, const fpg_forward_config* cfg, const fpg_release* releases,
                              size_t n_releases, const fpg_grid_domain* release_grid, size_t capacity,
                              size_t met_nx, size_t met_ny, size_t met_nz, const float* level_heights,
                              fpg_forward** out);
/* Waits for the context's stream and frees everything the driver owns; call
 * it before fpg_ctx_destroy of its context (as for every handle). */
fpg_status fpg_forward_destroy(fpg_forward* d);
/* has_remaining_steps (timeloop.rs:832-834): current time <= end. */
int32_t fpg_forward_has_remaining_steps(const fpg_forward* d);
int64_t fpg_forward_current_time(const fpg_forward* d);
/* run_timestep (timeloop.rs:915-1316).  Returns FPG_ERR_SIMULATION_COMPLETE
 * past the end, the release errors (InvalidBounds, OutOfGrid, StoreFull),
 * the bracket errors and the kernels' errors.  Work is queued on the
 * context's stream; the report's counts are host bookkeeping and need no
 * device wait (a compaction step waits for its active count, as the
 * reference's download_active_count does). */
fpg_status fpg_forward_run_timestep(fpg_forward* d, const fpg_met_bracket* met, const fpg_forcing* forcing,
                                    fpg_step_report* report);
/* finalize (timeloop.rs:1340-1346): waits for queued work. */
fpg_status fpg_forward_finalize(fpg_forward* d);
fpg_particles* fpg_forward_particles(fpg_forward* d);
/* accumulate_concentration_grid (timeloop.rs:888-896) into a caller grid. */
fpg_status fpg_forward_accumulate_grid(fpg_forward* d, fpg_grid* grid, uint32_t species_index,
                                       float mass_scale, const float* outheights, size_t n_outheights);

/* parse_timestamp_seconds (release/mod.rs:283-334): "YYYYMMDDHHMMSS". */
fpg_status fpg_parse_timestamp(const char* yyyymmddhhmmss, int64_t* seconds);

#ifdef __cplusplus
}
#endif

#endif /* FPG_DRIVER_H */
