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
    int32_t use_compaction;               /* is_compaction_enabled (timeloop.rs:506-513); FLEXPART_GPU_COMPACTION=1
                                             at create turns it on as well */
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

/* Met streaming, the device side of the reference's prefetching met reader
 * (io/grib2_async.rs:41-120 feeding MetTimeBracket): a ring of n_slots met
 * frames (u, v, w and surface cells) on the device, filled ahead of use on a
 * separate copy stream.  fpg_forward_prefetch_frame queues the copy of the
 * frame valid at time_seconds and returns without waiting (page-locked host
 * buffers, fpg_host_alloc, make the copy overlap the steps; device buffers
 * are copied on the device; either must stay unchanged until the frame is
 * used).  When run_timestep
 * meets a new bracket whose two frames are in the ring, it repacks them on
 * the device after their copies (no host copy, the bracket's host pointers
 * are not read); otherwise it uploads from the bracket's host pointers as
 * before.  A full ring evicts its least recently used frame outside the
 * current bracket (after the repack that read it), so with n_slots = 3 the
 * frame after the current bracket is prefetched once that bracket is in use
 * (after its first run_timestep).  n_slots >= 2; the ring is kept for the
 * driver's life.  Results do not depend on whether frames come from the
 * ring. */
fpg_status fpg_forward_met_ring(fpg_forward* d, uint32_t n_slots);
fpg_status fpg_forward_prefetch_frame(fpg_forward* d, int64_t time_seconds, const float* u, const float* v,
                                      const float* w, const fpg_surface_cell* surface);
/* Brackets served from the ring and from host pointers so far. */
fpg_status fpg_forward_met_ring_stats(const fpg_forward* d, uint64_t* ring_hits, uint64_t* host_uploads);

/* Per-section timing of one run_timestep: the reference's StepTimingReport
 * (timeloop.rs:398-467), measured here with CUDA events between the
 * sections on the device (ms) plus the host's time inside the call.
 * Sections: reorder, release (new particles uploaded), met bracket (ring
 * repack or host upload), PBL diagnostics, the fused step, compaction. */
typedef struct fpg_step_timing {
    uint64_t step_index;
    double sort_ms;
    double release_ms;
    double met_bracket_ms;
    double pbl_ms;
    double step_ms;
    double compaction_ms;
    double gpu_total_ms;           /* first to last section on the device */
    double host_call_ms;           /* host time inside run_timestep before the wait */
    double wall_ms;                /* host time of the call including the wait for the device */
} fpg_step_timing;

/* Turns the timing on or off (is_profiling_enabled, timeloop.rs:469-476:
 * also on when FLEXPART_GPU_PROFILE=1 at create time, which in addition
 * prints one summary line per step to stderr, as the reference does).
 * With timing on, every run_timestep waits for its device work to finish.
 * NVTX ranges mark every step and section whether timing is on or not. */
fpg_status fpg_forward_set_profiling(fpg_forward* d, int32_t on);
/* The reference's validation mode (is_validation_mode, timeloop.rs:480-494,
 * used at :1128-1155): each step runs advection, the per-slot Hanna records
 * (fpg_dispatch_hanna_params), the Langevin update from those records
 * (fpg_langevin_with_hanna) and deposition as separate passes instead of the
 * fused kernel.  The results are the fused kernel's, bit for bit.  Also on
 * when FLEXPART_GPU_VALIDATION=1 at create time.  Turning it on allocates
 * one 64-byte Hanna record per slot of the capacity. */
fpg_status fpg_forward_set_validation_mode(fpg_forward* d, int32_t on);
/* The timing of the last run_timestep made with timing on; NOT_READY if none. */
fpg_status fpg_forward_last_timing(const fpg_forward* d, fpg_step_timing* out);

/* ------------------------------------------------------------------------
 * Backward (receptor) mode: BackwardTimeLoopDriver
 * (src/simulation/timeloop.rs:1433-1909).
 *
 * Receptors release their particles at the start time (later than the end
 * time); the clock runs backward by timestep_seconds per step; each step is
 * the fused step with advection at -dt and turbulence and deposition at +dt
 * (timeloop.rs:1724-1768), the Philox counter advancing by capacity x
 * blocks; after the step, the active particles inside each source region
 * are counted and their species-0 mass summed (collect_source_collections,
 * timeloop.rs:1865-1894) by one device pass.
 * ---------------------------------------------------------------------- */

/* BackwardReceptorConfig (timeloop.rs:150-163): a point release at (lon, lat,
 * z_m) of particle_count particles carrying mass_kg in all. */
typedef struct fpg_receptor_release {
    double lon, lat, z_m;
    uint64_t particle_count;
    double mass_kg;
} fpg_receptor_release;

/* BackwardSourceRegionConfig (timeloop.rs:170-197): inclusive bounds;
 * a particle's lon = xlon0 + (cell_x + pos_x) * dx in double, lat likewise. */
typedef struct fpg_source_region {
    double lon_min, lon_max;
    double lat_min, lat_max;
    double z_min_m, z_max_m;
} fpg_source_region;

/* BackwardSourceCollection (timeloop.rs:201-206).  total_mass_kg is the sum
 * in double rounded to float (the reference adds floats in slot order, whose
 * rounding depends on that order); total_mass_kg_f64 is the double sum. */
typedef struct fpg_source_collection {
    uint64_t hit_count;
    float total_mass_kg;
    float pad;
    double total_mass_kg_f64;
} fpg_source_collection;

/* BackwardTimeLoopConfig (timeloop.rs:226-251). */
typedef struct fpg_backward_config {
    int64_t start_seconds, end_seconds;   /* start >= end; both inclusive */
    int64_t timestep_seconds;             /* > 0: the step magnitude */
    int32_t clamp_time_bounds;            /* TimeBoundsBehavior: 1 Clamp, 0 Strict */
    float x_grid_per_meter, y_grid_per_meter, z_grid_per_meter;
    fpg_pbl_options pbl_options;
    float dry_reference_height_m;         /* 15 m */
    uint32_t philox_key[2];
    uint32_t initial_philox_counter[4];
    uint32_t n_substeps;                  /* 4 (timeloop.rs:1744) */
    float min_height_m;                   /* 0.01 (timeloop.rs:1745) */
} fpg_backward_config;

/* The reference's defaults (timeloop.rs:253-270, the step of :1741-1746). */
void fpg_backward_config_default(fpg_backward_config* cfg);

typedef struct fpg_backward fpg_backward;

/* BackwardTimeLoopDriver::new (timeloop.rs:1497-1571) with
 * validate_backward_config (:1974-2073): FPG_ERR_INVALID_BACKWARD_TIME_RANGE,
 * FPG_ERR_INVALID_TIME_STEP, FPG_ERR_INVALID_REFERENCE_HEIGHT,
 * FPG_ERR_MISSING_RECEPTORS, FPG_ERR_INVALID_RECEPTOR (lon outside
 * [-180, 180], lat outside [-90, 90], z < 0 or not finite, count 0, mass
 * <= 0 or not finite), FPG_ERR_INVALID_SOURCE_BOUNDS (min > max). */
fpg_status fpg_backward_create(fpg_ctx* ctx, const fpg_backward_config* cfg, const fpg_receptor_release* receptors,
                               size_t n_receptors, const fpg_source_region* regions, size_t n_regions,
                               const fpg_grid_domain* release_grid, size_t capacity, size_t met_nx, size_t met_ny,
                               size_t met_nz, const float* level_heights, fpg_backward** out);
fpg_status fpg_backward_destroy(fpg_backward* d);
/* has_remaining_steps (timeloop.rs:1573-1577): current time >= end. */
int32_t fpg_backward_has_remaining_steps(const fpg_backward* d);
int64_t fpg_backward_current_time(const fpg_backward* d);
/* run_timestep (timeloop.rs:1598-1821): release, alpha, bracket, PBL, the
 * step at -dt / +dt, then the source collections (n_regions entries, may be
 * NULL); waits for the device, as the reference does every backward step. */
fpg_status fpg_backward_run_timestep(fpg_backward* d, const fpg_met_bracket* met, const fpg_forcing* forcing,
                                     fpg_step_report* report, fpg_source_collection* collections);
fpg_particles* fpg_backward_particles(fpg_backward* d);
/* The separated passes of fpg_forward_set_validation_mode for the backward
 * step, the path the reference's backward driver always takes
 * (timeloop.rs:1433-1437); the same bits as the fused kernel. */
fpg_status fpg_backward_set_validation_mode(fpg_backward* d, int32_t on);

/* ------------------------------------------------------------------------
 * Batched ensemble: many independent release scenarios stepped together.
 *
 * No counterpart in the reference, which runs one scenario per driver.  Each
 * scenario is what one ForwardTimeLoopDriver with one release, capacity =
 * its particle_count, its own Philox key and initial counter would compute
 * (the same release lattice, slots, counters and kernels), so its particles
 * come out bit for bit as in a plain run of it alone.  All scenarios share
 * one met frame ring and one global clock; their particles sit in one
 * structure-of-arrays population, each scenario in a 256-slot-aligned
 * segment.  One step is a CUDA graph of device-side kernels (clock and
 * release bookkeeping, bracket repack when it changes, per-cell PBL and wet
 * forcing, release of new particles, one persistent launch over all
 * scenarios' tiles from a work queue, per-scenario grids at output steps,
 * counter advance), so the host only launches the graph.
 * ---------------------------------------------------------------------- */
typedef struct fpg_batch_scenario {
    fpg_release release;
    uint32_t key[2];
    uint32_t counter[4];
} fpg_batch_scenario;

typedef struct fpg_batch_config {
    int64_t start_seconds, end_seconds, timestep_seconds;
    int64_t frame_seconds;          /* frames k at start + k*frame_seconds, cycled */
    uint32_t n_frames;
    float x_grid_per_meter, y_grid_per_meter, z_grid_per_meter;
    fpg_pbl_options pbl_options;
    float dry_reference_height_m;
    float dry_velocity_m_s;         /* 0: no dry deposition */
    float rho_grad_over_rho;
    uint32_t n_substeps;
    float min_height_m;
    int32_t wet_from_precipitation; /* per-cell wet forcing from each bracket's t0 precipitation */
    float wet_gas_a, wet_gas_b;
    fpg_grid_domain release_grid;
    uint32_t out_nx, out_ny, out_nz;
    const float* outheights;        /* out_nz heights (copied at create) */
    uint32_t output_every_steps;    /* grids at steps k with (k+1) % every == 0; 0: never */
} fpg_batch_config;

typedef struct fpg_batch fpg_batch;

/* 1 <= n_scenarios <= 65535; every particle_count and release window below
 * 2^32 (FPG_ERR_VALUE_TOO_LARGE); FPG_ERR_OUT_OF_GRID when a scenario's
 * release lattice leaves release_grid, as the release manager reports it at
 * injection (release/mod.rs:41). */
fpg_status fpg_batch_create(fpg_ctx* ctx, const fpg_batch_config* cfg, const fpg_batch_scenario* scenarios,
                            size_t n_scenarios, size_t met_nx, size_t met_ny, size_t met_nz,
                            const float* level_heights, fpg_batch** out);
fpg_status fpg_batch_destroy(fpg_batch* b);
/* Frame k of the met ring: u, v, w (nx*ny*nz, reference layout), surface
 * cells (nx*ny) and large-scale precipitation [mm/h] (nx*ny, may be NULL). */
fpg_status fpg_batch_upload_frame(fpg_batch* b, uint32_t k, const float* u, const float* v, const float* w,
                                  const fpg_surface_cell* surface, const float* precipitation_mm_h);
/* Runs n_steps steps (fewer if the end time comes first): each step is one
 * replay of the captured graph when use_graph is non-zero (the graph is
 * captured on the first call), else the same kernels launched one by one.
 * Returns FPG_ERR_SIMULATION_COMPLETE when no step is left. */
fpg_status fpg_batch_run(fpg_batch* b, uint32_t n_steps, int32_t use_graph);
/* The same steps with one plain fused-step launch per scenario per step
 * (sequential launches, no graph): the comparison the batching is measured
 * against.  Bit-identical results. */
fpg_status fpg_batch_run_sequential(fpg_batch* b, uint32_t n_steps);
/* Steps taken so far; slot range of scenario s; the whole population. */
uint64_t fpg_batch_steps_done(const fpg_batch* b);
fpg_status fpg_batch_scenario_slots(const fpg_batch* b, size_t s, size_t* first_slot, size_t* count);
fpg_particles* fpg_batch_particles(fpg_batch* b);
/* Per-scenario grids of the last output step: n_scenarios * out cells each
 * (scenario-major), u32 counts and scaled masses (scale 1e6). */
fpg_status fpg_batch_download_grids(fpg_batch* b, uint32_t* counts, uint32_t* mass_scaled);
/* Device-side error flags (1: a release fell outside the grid). */
fpg_status fpg_batch_errors(fpg_batch* b, int32_t* flags);

/* Launch shapes of the particle pass (fpg_batch_tuning, fpg.h): threads per
 * CTA, CTAs resident per SM the kernel is compiled for (its register
 * budget), and particles per thread in one work item (a work item is
 * block_threads * particles_per_thread consecutive slots of one scenario),
 * which persistent CTAs pull from a counter.  particles_per_thread 0 is the
 * non-persistent pass: one CTA per item of block_threads slots, one slot per
 * thread, launched over all items.  step_ms is the particle pass's time
 * measured by the tuner (0 when set by hand).
 * The compiled launch shapes: writes up to max of them, returns their count. */
uint32_t fpg_batch_tuning_candidates(fpg_batch_tuning* out, uint32_t max);
/* Times the next step's particle pass under every compiled shape (best of
 * reps), each from the same snapshot of the live state, restores the state
 * and keeps the fastest shape.  Results are identical under every shape.
 * Needs device memory for one copy of the population.  results (up to
 * max_results entries, candidate order) and best may be NULL.  Call it once
 * the population is representative (after some steps), or tune a copy of the
 * run and pass the choice to fpg_batch_set_tuning. */
fpg_status fpg_batch_autotune(fpg_batch* b, uint32_t reps, fpg_batch_tuning* results, uint32_t max_results,
                              fpg_batch_tuning* best);
/* Selects a compiled shape (FPG_ERR_INVALID_ARGUMENT if none matches). */
fpg_status fpg_batch_set_tuning(fpg_batch* b, const fpg_batch_tuning* tuning);
fpg_status fpg_batch_get_tuning(const fpg_batch* b, fpg_batch_tuning* tuning);

/* parse_timestamp_seconds (release/mod.rs:283-334): "YYYYMMDDHHMMSS". */
fpg_status fpg_parse_timestamp(const char* yyyymmddhhmmss, int64_t* seconds);

#ifdef __cplusplus
}
#endif

#endif /* FPG_DRIVER_H */
