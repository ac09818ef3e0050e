/*
 * fpg.h — C ABI of the B200 (sm_100a) backend for the flexpart-gpu
 * per-particle timestep.
 *
 * The reference crate (Improba/flexpart-gpu, Rust + WGSL via wgpu) drives the
 * step from ForwardTimeLoopDriver::run_timestep (src/simulation/timeloop.rs:915-1316)
 * through a set of `encode_*_gpu_with_kernel` functions that each append one
 * compute pass to a wgpu command encoder.  Every function below is the
 * replacement for one of those seam functions (cited beside it), or for a
 * buffer owner method it needs.  The conventions:
 *
 *  - every call returns fpg_status (int32_t); 0 is success and the negative
 *    codes mirror the reference's thiserror enums (cited at fpg_status);
 *  - handles own device memory; callers own every host array they pass;
 *  - calls are ordered on a CUDA stream: `stream` is a cudaStream_t passed as
 *    void*, NULL meaning the context's own stream.  A call that returns data
 *    to the host synchronises that stream first;
 *  - one context per host thread; a context is bound to one device;
 *  - no exceptions and no C++ or torch types cross this boundary.
 *
 * Particle state lives on the device as structure-of-arrays (one array per
 * field).  The 96-byte fpg_particle record is only the exchange format of
 * upload/download, byte-compatible with the reference's #[repr(C)] Particle
 * (src/particles/mod.rs:76-168).
 */
#ifndef FPG_H
#define FPG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FPG_ABI_VERSION 1

/* src/particles/mod.rs:18 (MAX_SPECIES) and :21 (FLAG_ACTIVE). */
#define FPG_MAX_SPECIES 4
#define FPG_FLAG_ACTIVE 1u
/* Upper bound on vertical wind levels and output heights held on chip.  The
 * reference caps both at 16 (src/physics/advection.rs:20,
 * src/gpu/gridding.rs:85); this backend generalises the same scans. */
#define FPG_MAX_LEVELS 256

typedef int32_t fpg_status;
enum {
    FPG_OK = 0,
    FPG_ERR_INVALID_ARGUMENT = -1,   /* null handle / pointer, bad enum */
    FPG_ERR_INVALID_TIME_STEP = -2,  /* InvalidTimeStep: gpu/langevin_fused.rs:119, gpu/advection.rs, gpu/deposition.rs */
    FPG_ERR_ZERO_SHAPE = -3,         /* ZeroShape / ZeroPblShape / ZeroGridShape: gpu/gridding.rs:226, gpu/langevin_fused.rs:122, gpu/pbl.rs:90 */
    FPG_ERR_VALUE_TOO_LARGE = -4,    /* ValueTooLarge (does not fit u32): gpu/langevin_fused.rs:124 */
    FPG_ERR_LENGTH_MISMATCH = -5,    /* LengthMismatch: gpu/deposition.rs:328, gpu/wet_deposition.rs:381 */
    FPG_ERR_INVALID_SPECIES = -6,    /* InvalidSpeciesIndex: gpu/gridding.rs:228 */
    FPG_ERR_INVALID_MASS_SCALE = -7, /* InvalidMassScale: gpu/gridding.rs:233 */
    FPG_ERR_INVALID_REFERENCE_HEIGHT = -8, /* InvalidReferenceHeight: gpu/deposition.rs:340 */
    FPG_ERR_STORE_FULL = -9,         /* ParticleError::StoreFull: particles/mod.rs:516 */
    FPG_ERR_SHAPE_MISMATCH = -10,    /* ShapeMismatch: gpu/pbl.rs:92 */
    FPG_ERR_NOT_READY = -11,         /* a required buffer (met bracket, PBL) was never uploaded */
    FPG_ERR_INVALID_BRACKET = -12,   /* TemporalInterpolationError::InvalidTimeBracket: simulation/timeloop.rs:2093 */
    FPG_ERR_OUTSIDE_BRACKET = -13,   /* TemporalInterpolationError::TargetOutsideBracket: simulation/timeloop.rs:2104 */
    FPG_ERR_SIMULATION_COMPLETE = -14, /* TimeLoopError::SimulationComplete: simulation/timeloop.rs:921 */
    FPG_ERR_INVALID_BOUNDS = -15,    /* ReleaseError::InvalidBounds: release/mod.rs:33 */
    FPG_ERR_OUT_OF_GRID = -16,       /* ReleaseError::OutOfGridDomain: release/mod.rs:41 */
    FPG_ERR_TOO_MANY_LEVELS = -17,   /* more than FPG_MAX_LEVELS heights */
    FPG_ERR_INVALID_TIME_RANGE = -18, /* TimeLoopError::InvalidTimeRange: simulation/timeloop.rs:1935 */
    FPG_ERR_INVALID_BACKWARD_TIME_RANGE = -19, /* TimeLoopError::InvalidBackwardTimeRange: simulation/timeloop.rs:1978 */
    FPG_ERR_MISSING_RECEPTORS = -20, /* TimeLoopError::MissingReceptors: simulation/timeloop.rs:1994 */
    FPG_ERR_INVALID_RECEPTOR = -21,  /* TimeLoopError::InvalidReceptor: simulation/timeloop.rs:2006-2046 */
    FPG_ERR_INVALID_SOURCE_BOUNDS = -22, /* TimeLoopError::InvalidSourceBounds: simulation/timeloop.rs:2049-2073 */
    FPG_ERR_NON_STOCHASTIC_COLUMN = -23, /* ConvectionError::NonStochasticColumn: physics/convection.rs:196-218 */
    FPG_ERR_TOO_FEW_LEVELS = -24,    /* ConvectionError::TooFewLevels: physics/convection.rs:86-90 */
    FPG_ERR_NON_MONOTONIC_INTERFACES = -25, /* ConvectionError::NonMonotonicInterfaces: physics/convection.rs:92-98 */
    FPG_ERR_INVALID_BOUNDARY_LAYER_HEIGHT = -26, /* ConvectionError::InvalidBoundaryLayerHeight: physics/convection.rs:100-104 */
    FPG_ERR_CUDA = -100,             /* any CUDA runtime error (see fpg_last_cuda_error) */
    FPG_ERR_OUT_OF_MEMORY = -101,
    FPG_ERR_NO_DEVICE = -102
};

/* Returns a static string for a status code. */
const char* fpg_status_string(fpg_status status);
/* Last CUDA error code (cudaError_t as int) seen by this thread, 0 if none. */
int32_t fpg_last_cuda_error(void);
/* FPG_ABI_VERSION of the loaded library. */
int32_t fpg_abi_version(void);

/* ------------------------------------------------------------------------
 * Exchange records
 * ---------------------------------------------------------------------- */

/* One particle, 96 bytes: src/particles/mod.rs:76-168 field for field. */
typedef struct fpg_particle {
    float pos_x, pos_y, pos_z;      /* fractional cell offsets, height [m] */
    int32_t cell_x, cell_y;
    uint32_t flags;                 /* bit 0 = active */
    float mass[FPG_MAX_SPECIES];
    float vel_u, vel_v, vel_w;
    float turb_u, turb_v, turb_w;
    int32_t time, timestep, time_mem, time_split;
    int32_t release_point, class_id, cbt;
    uint32_t pad0;
} fpg_particle;

/* Packed surface input of one met cell, 48 bytes: SurfaceCellInputGpu,
 * src/gpu/pbl.rs:35-50 (cells ordered i*ny + j). */
typedef struct fpg_surface_cell {
    float surface_pressure_pa;
    float temperature_2m_k;
    float u10_ms, v10_ms;
    float surface_stress_n_m2;
    float sensible_heat_flux_w_m2;
    float solar_radiation_w_m2;
    float mixing_height_m;           /* <= 0 or non-finite: unavailable */
    float friction_velocity_ms;      /* <= 0 or non-finite: unavailable */
    float inv_obukhov_length_per_m;  /* |1/L| < 1e-5 or non-finite: unavailable */
    float pad0, pad1;
} fpg_surface_cell;

/* PblComputationOptions, src/io/pbl_params.rs:35-68 (fields the GPU path
 * reads: src/shaders/pbl_diagnostics.wgsl:46-59). */
typedef struct fpg_pbl_options {
    float roughness_length_m;              /* default 0.1 */
    float wind_reference_height_m;         /* default 10 */
    float heat_flux_neutral_threshold_w_m2;/* default 1 */
    float fallback_mixing_height_m;        /* default 800 */
    float hmix_min_m;                      /* default 100 (lib.rs:44) */
    float hmix_max_m;                      /* default 4500 (lib.rs:46) */
} fpg_pbl_options;

/* ------------------------------------------------------------------------
 * Context
 * ---------------------------------------------------------------------- */
typedef struct fpg_ctx fpg_ctx;

/* GpuContext::new (src/gpu/mod.rs:163-208): binds `device`, creates a stream. */
fpg_status fpg_ctx_create(int32_t device, fpg_ctx** out);
/* Every handle created on a context must be destroyed before the context. */
fpg_status fpg_ctx_destroy(fpg_ctx* ctx);
/* The context's stream as a cudaStream_t. */
void* fpg_ctx_stream(fpg_ctx* ctx);
/* device.poll(Maintain::Wait): waits for all work queued on `stream`. */
fpg_status fpg_ctx_synchronize(fpg_ctx* ctx, void* stream);
/* Number of kernels this context has launched since creation (all entry
 * points, graph replays counted per kernel node). */
uint64_t fpg_ctx_kernel_launches(fpg_ctx* ctx);

/* Plain device buffers for callers without a CUDA allocator of their own
 * (the role wgpu::Buffer plays for the reference's per-slot forcing and
 * probability arrays, gpu/deposition.rs, gpu/wet_deposition.rs).
 * fpg_memcpy kind: 0 host->device, 1 device->host (returns after the copy),
 * 2 device->device. */
fpg_status fpg_device_alloc(fpg_ctx* ctx, size_t bytes, void** out);
fpg_status fpg_device_free(fpg_ctx* ctx, void* ptr);
fpg_status fpg_memcpy(fpg_ctx* ctx, void* dst, const void* src, size_t bytes, int32_t kind, void* stream);
fpg_status fpg_memset(fpg_ctx* ctx, void* dst, int32_t value, size_t bytes, void* stream);
/* Page-locked host memory: copies from it to the device run asynchronously
 * and overlap kernels (fpg_forward_prefetch_frame streams met frames from
 * such buffers). */
fpg_status fpg_host_alloc(fpg_ctx* ctx, size_t bytes, void** out);
fpg_status fpg_host_free(fpg_ctx* ctx, void* ptr);

/* ------------------------------------------------------------------------
 * Particles (ParticleBuffers, src/gpu/buffers.rs:377-510)
 * ---------------------------------------------------------------------- */
typedef struct fpg_particles fpg_particles;

/* ParticleBuffers::from_store on an empty store: `capacity` zeroed
 * (inactive) slots; dispatch count = capacity. */
fpg_status fpg_particles_create(fpg_ctx* ctx, size_t capacity, fpg_particles** out);
fpg_status fpg_particles_destroy(fpg_particles* p);
size_t fpg_particles_capacity(const fpg_particles* p);
/* ParticleBuffers::particle_count / set_dispatch_count / reset_dispatch_count
 * (buffers.rs:408-436): slots [0, count) are processed by every kernel. */
size_t fpg_particles_dispatch_count(const fpg_particles* p);
fpg_status fpg_particles_set_dispatch_count(fpg_particles* p, size_t count);
/* upload_particle_slots for the contiguous slots [first, first+count)
 * (buffers.rs:464-492). `records` is host memory. */
fpg_status fpg_particles_upload(fpg_particles* p, size_t first, size_t count,
                                const fpg_particle* records, void* stream);
/* upload_particle_slots for an arbitrary slot list. */
fpg_status fpg_particles_upload_slots(fpg_particles* p, const uint32_t* slots, size_t count,
                                     const fpg_particle* records, void* stream);
/* download_particles (buffers.rs:111-163) for [first, first+count). */
fpg_status fpg_particles_download(fpg_particles* p, size_t first, size_t count,
                                  fpg_particle* out, void* stream);

/* Field ids of the structure-of-arrays state, for direct device access. */
enum {
    FPG_FIELD_POS_X = 0, FPG_FIELD_POS_Y, FPG_FIELD_POS_Z,
    FPG_FIELD_CELL_X, FPG_FIELD_CELL_Y, FPG_FIELD_FLAGS,
    FPG_FIELD_MASS0, FPG_FIELD_MASS1, FPG_FIELD_MASS2, FPG_FIELD_MASS3,
    FPG_FIELD_VEL_U, FPG_FIELD_VEL_V, FPG_FIELD_VEL_W,
    FPG_FIELD_TURB_U, FPG_FIELD_TURB_V, FPG_FIELD_TURB_W,
    FPG_FIELD_TIME, FPG_FIELD_TIMESTEP, FPG_FIELD_TIME_MEM, FPG_FIELD_TIME_SPLIT,
    FPG_FIELD_RELEASE_POINT, FPG_FIELD_CLASS, FPG_FIELD_CBT,
    FPG_FIELD_COUNT
};
/* Device pointer of one 4-byte-per-slot field array (capacity elements). */
void* fpg_particles_field(fpg_particles* p, int32_t field);
/* Copy `count` elements of one field between host and device
 * (to_device != 0: host -> device).  Host memory may be pinned or pageable. */
fpg_status fpg_particles_copy_field(fpg_particles* p, int32_t field, size_t first, size_t count,
                                    void* host, int32_t to_device, void* stream);

/* ------------------------------------------------------------------------
 * Dual-time wind bracket (DualWindBuffers, src/gpu/buffers.rs:801-950)
 * ---------------------------------------------------------------------- */
typedef struct fpg_met fpg_met;

fpg_status fpg_met_create(fpg_ctx* ctx, size_t nx, size_t ny, size_t nz, fpg_met** out);
fpg_status fpg_met_destroy(fpg_met* m);
/* DualWindBuffers::upload_t0 / upload_t1: `which` 0 = t0, 1 = t1.  u, v, w
 * are host arrays of nx*ny*nz floats in the reference layout
 * ((ix*ny)+iy)*nz+iz (z fastest, buffers.rs:229-235). */
fpg_status fpg_met_upload_frame(fpg_met* m, int32_t which, const float* u, const float* v,
                                const float* w, void* stream);
/* Same from device arrays (already resident frames, e.g. a frame ring). */
fpg_status fpg_met_upload_frame_device(fpg_met* m, int32_t which, const float* u_dev,
                                       const float* v_dev, const float* w_dev, void* stream);
/* Both frames of a new bracket from device arrays in one pass
 * (upload_dual_wind_if_bracket_changed, src/simulation/timeloop.rs:1378-1402,
 * uploads t0 and t1 together): the same bracket as two
 * fpg_met_upload_frame_device calls, writing each node whole. */
fpg_status fpg_met_upload_bracket_device(fpg_met* m, const float* u0_dev, const float* v0_dev,
                                         const float* w0_dev, const float* u1_dev, const float* v1_dev,
                                         const float* w1_dev, void* stream);
/* VelocityToGridScale::level_heights_m (advection.rs:31-41): heights [m] of
 * the nz wind levels.  All-zero (top <= 0) selects the legacy mode where
 * pos_z is a level index.  n must equal nz (n <= FPG_MAX_LEVELS). */
fpg_status fpg_met_set_level_heights(fpg_met* m, const float* heights, size_t n);

/* ------------------------------------------------------------------------
 * PBL fields (PblBuffers, src/gpu/buffers.rs:955-1060) and per-cell surface
 * input (SurfaceFieldBuffer, src/gpu/pbl.rs:142-240)
 * ---------------------------------------------------------------------- */
typedef struct fpg_pbl fpg_pbl;
typedef struct fpg_surface fpg_surface;

fpg_status fpg_pbl_create(fpg_ctx* ctx, size_t nx, size_t ny, fpg_pbl** out);
fpg_status fpg_pbl_destroy(fpg_pbl* pbl);
/* PblBuffers::upload_state: host arrays of nx*ny floats (i*ny + j). */
fpg_status fpg_pbl_upload(fpg_pbl* pbl, const float* ustar, const float* wstar, const float* hmix,
                          const float* oli, const float* sshf, const float* ssr,
                          const float* surfstr, void* stream);
/* Reads the seven PBL fields back (any pointer may be NULL). */
fpg_status fpg_pbl_download(fpg_pbl* pbl, float* ustar, float* wstar, float* hmix, float* oli,
                            float* sshf, float* ssr, float* surfstr, void* stream);

fpg_status fpg_surface_create(fpg_ctx* ctx, size_t nx, size_t ny, fpg_surface** out);
fpg_status fpg_surface_destroy(fpg_surface* s);
/* SurfaceFieldBuffer::upload of one frame: `which` 0 = t0, 1 = t1.  The
 * device lerps the two frames (io/temporal.rs:122,417-420) inside
 * fpg_pbl_diagnostics, so a bracket is uploaded once, not every step.
 * `cells` may be host or device memory (unified addressing). */
fpg_status fpg_surface_upload(fpg_surface* s, int32_t which, const fpg_surface_cell* cells,
                              void* stream);

/* encode_pbl_diagnostics_gpu_with_kernel (src/gpu/pbl.rs:367) preceded by
 * interpolate_surface_fields_linear (src/io/temporal.rs:122): per met cell,
 * lerp the t0/t1 surface frames by `alpha` (0 uses t0 only, 1 t1 only, as the
 * reference's early returns do), then compute u*, w*, hmix, 1/L into `pbl`.
 * Errors: ZeroShape, ShapeMismatch. */
fpg_status fpg_pbl_diagnostics(fpg_ctx* ctx, const fpg_surface* surface, float alpha,
                               const fpg_pbl_options* options, fpg_pbl* pbl, void* stream);

/* ------------------------------------------------------------------------
 * Per-cell deposition forcing (2-D, i*ny + j)
 * ---------------------------------------------------------------------- */
typedef struct fpg_cellfield fpg_cellfield;
fpg_status fpg_cellfield_create(fpg_ctx* ctx, size_t nx, size_t ny, fpg_cellfield** out);
fpg_status fpg_cellfield_destroy(fpg_cellfield* f);
/* Uploads per-cell (lambda [1/s], precipitating fraction [-]) pairs. */
fpg_status fpg_cellfield_upload(fpg_cellfield* f, const float* lambda, const float* fraction,
                                void* stream);
/* Derives the per-cell wet forcing from precipitation on the device:
 * wet_precipitation_state (src/physics/wet_scavenging.rs:179-207) gives the
 * precipitating fraction and sub-grid rate, then the below-cloud gas
 * coefficient a * prec^b (wet_scavenging.rs:213-225).  Inputs are host or
 * device arrays of large-scale and convective precipitation [mm/h] and
 * cloud cover [-] (any may be NULL = 0, cloud cover NULL = 1). */
fpg_status fpg_cellfield_from_precipitation(fpg_cellfield* f, const float* lsp_mm_h,
                                            const float* convp_mm_h, const float* cloud_cover,
                                            float gas_coefficient_a, float gas_exponent_b,
                                            void* stream);

/* ------------------------------------------------------------------------
 * The fused step
 * ---------------------------------------------------------------------- */
enum { /* how a deposition input is supplied */
    FPG_FORCING_NONE = 0,         /* process skipped (ParticleForcingField::Uniform(0)) */
    FPG_FORCING_UNIFORM = 1,      /* one scalar for all slots */
    FPG_FORCING_PER_PARTICLE = 2, /* device arrays indexed by slot (the reference seam) */
    FPG_FORCING_PER_CELL = 3      /* fpg_cellfield looked up at the particle's nearest cell */
};

enum { /* stages of fpg_step (bit mask) */
    FPG_STAGE_ADVECT = 1u,     /* advection_dual_wind.wgsl */
    FPG_STAGE_TURBULENCE = 2u, /* langevin_fused.wgsl */
    FPG_STAGE_DRY = 4u,        /* dry_deposition.wgsl */
    FPG_STAGE_WET = 8u,        /* wet_deposition.wgsl */
    FPG_STAGE_ALL = 15u
};

typedef struct fpg_step_params {
    uint32_t stages;            /* FPG_STAGE_* mask */
    float alpha;                /* temporal weight of t1; clamped to [0,1] (gpu/advection.rs:639) */
    float dt_seconds;           /* advection dt (may be negative: backward mode) */
    float turb_dt_seconds;      /* Langevin / deposition dt (> 0 for turbulence) */
    float x_grid_per_meter;     /* VelocityToGridScale (physics/advection.rs:36-41) */
    float y_grid_per_meter;
    float z_grid_per_meter;
    uint32_t n_substeps;        /* LangevinStep::n_substeps (physics/langevin.rs:46), 4 in production */
    float min_height_m;         /* LangevinStep::min_height_m, 0.01 in production */
    float rho_grad_over_rho;    /* ForwardStepForcing::rho_grad_over_rho */
    uint32_t key[2];            /* Philox key */
    uint32_t counter[4];        /* Philox base counter of this step */
    float dry_reference_height_m; /* DryDepositionStepParams::reference_height_m (15 m) */
    int32_t dry_mode;           /* FPG_FORCING_* */
    float dry_velocity_m_s;     /* UNIFORM value */
    const float* dry_velocity_dev;   /* PER_PARTICLE device array (capacity) */
    float* dry_probability_dev;      /* optional device output (capacity), NULL = not written */
    int32_t wet_mode;           /* FPG_FORCING_* */
    float wet_lambda_s_inv;     /* UNIFORM values */
    float wet_fraction;
    const float* wet_lambda_dev;     /* PER_PARTICLE device arrays */
    const float* wet_fraction_dev;
    const fpg_cellfield* wet_cells;  /* PER_CELL */
    float* wet_probability_dev;      /* optional device output (capacity) */
} fpg_step_params;

/* Fills `params` with the production defaults of the forward loop
 * (simulation/timeloop.rs:1062-1113): all stages, alpha 0, n_substeps 4,
 * min height 0.01 m, href 15 m, no deposition forcing, scales 1. */
void fpg_step_params_default(fpg_step_params* params);

/* A launch shape of a particle kernel: CUDA block size, resident blocks per
 * SM the kernel is compiled for, particles per thread, and the time a tuner
 * measured for it (0 when set by hand).  The batched step (fpg_driver.h)
 * and the fused step share it. */
typedef struct fpg_batch_tuning {
    uint32_t block_threads;
    uint32_t min_blocks_per_sm;
    uint32_t particles_per_thread;
    float step_ms;
} fpg_batch_tuning;

/* One fused pass over slots [0, dispatch_count) of `particles`, replacing, in
 * this order:
 *   encode_advection_dual_wind_gpu_with_kernel (src/gpu/advection.rs:605),
 *   encode_langevin_fused_gpu                  (src/gpu/langevin_fused.rs:133),
 *   encode_dry_deposition_probability_gpu_with_kernel (src/gpu/deposition.rs:315),
 *   encode_wet_deposition_probability_gpu_with_kernel (src/gpu/wet_deposition.rs:368).
 * Each particle is read once and written once.  `next_counter` receives the
 * Philox counter for the next step (langevin_fused.rs:229-233; unchanged when
 * the dispatch count is 0 or turbulence is off).  `met` may be NULL when
 * advection is off, `pbl` when turbulence is off.
 * Errors: InvalidTimeStep (non-finite dt; turbulence dt <= 0), ZeroShape,
 * ValueTooLarge, InvalidReferenceHeight, NotReady. */
fpg_status fpg_step(fpg_ctx* ctx, fpg_particles* particles, const fpg_met* met,
                    const fpg_pbl* pbl, const fpg_step_params* params,
                    uint32_t next_counter[4], void* stream);

/* The four seam functions one at a time (same kernel, one stage). */
/* Launch shapes of fpg_step: the counterpart of the reference's workgroup
 * size autotune (auto_tune_key_kernels, src/gpu/workgroup.rs:377-440, which
 * times each candidate workgroup size of the key kernels and keeps the
 * fastest), over CUDA block size, resident blocks per SM and particles per
 * thread.  Every shape gives the same results bit for bit.  The shape is a
 * setting of the context (shape 0, <256, 5, 1>, until changed).
 * fpg_step_tuning_candidates writes up to `max` compiled shapes and returns
 * their count.  fpg_step_autotune times one fpg_step of `params` under every
 * shape (best of `reps`), each from the same snapshot of the particle state,
 * restores the state, keeps the fastest shape in the context and returns it
 * in `best`; it needs device memory for one copy of the particle arrays, and
 * the Philox counter is not advanced.  `results` (candidate order) and `best`
 * may be NULL.  fpg_step_set_tuning selects a compiled shape
 * (FPG_ERR_INVALID_ARGUMENT if none matches). */
uint32_t fpg_step_tuning_candidates(fpg_batch_tuning* out, uint32_t max);
fpg_status fpg_step_autotune(fpg_ctx* ctx, fpg_particles* particles, const fpg_met* met, const fpg_pbl* pbl,
                             const fpg_step_params* params, uint32_t reps, fpg_batch_tuning* results,
                             uint32_t max_results, fpg_batch_tuning* best, void* stream);
fpg_status fpg_step_set_tuning(fpg_ctx* ctx, const fpg_batch_tuning* tuning);
fpg_status fpg_step_get_tuning(const fpg_ctx* ctx, fpg_batch_tuning* tuning);

fpg_status fpg_advect_dual_wind(fpg_ctx* ctx, fpg_particles* particles, const fpg_met* met,
                                float alpha, float dt_seconds, float x_grid_per_meter,
                                float y_grid_per_meter, float z_grid_per_meter, void* stream);
fpg_status fpg_langevin_fused(fpg_ctx* ctx, fpg_particles* particles, const fpg_pbl* pbl,
                              float dt_seconds, float rho_grad_over_rho, uint32_t n_substeps,
                              float min_height_m, const uint32_t key[2],
                              const uint32_t base_counter[4], uint32_t next_counter[4],
                              void* stream);
/* vdep_dev / prob_dev are device arrays of dispatch_count floats (prob may be NULL). */
fpg_status fpg_dry_deposition(fpg_ctx* ctx, fpg_particles* particles, const float* vdep_dev,
                              float dt_seconds, float reference_height_m, float* prob_dev,
                              void* stream);
fpg_status fpg_wet_deposition(fpg_ctx* ctx, fpg_particles* particles, const float* lambda_dev,
                              const float* fraction_dev, float dt_seconds, float* prob_dev,
                              void* stream);

/* ------------------------------------------------------------------------
 * Concentration gridding (src/gpu/gridding.rs:255-420)
 * ---------------------------------------------------------------------- */
typedef struct fpg_grid fpg_grid;

fpg_status fpg_grid_create(fpg_ctx* ctx, size_t nx, size_t ny, size_t nz, fpg_grid** out);
fpg_status fpg_grid_destroy(fpg_grid* g);
/* dispatch_concentration_gridding_gpu (gridding.rs:255-406): clears the grid,
 * then bins active slots [0, dispatch_count) into (clamp(cell_x),
 * clamp(cell_y), level(pos_z)) adding 1 to the count and
 * u32(mass*scale + 0.5) to the mass grid (concentration_gridding.wgsl:284-345).
 * `outheights` has nz entries (or NULL = all zero: floor(pos_z) levels).
 * Integer sums: the result does not depend on thread order.
 * Errors: ZeroShape, InvalidSpeciesIndex, InvalidMassScale, ValueTooLarge. */
fpg_status fpg_grid_accumulate(fpg_ctx* ctx, const fpg_particles* particles, fpg_grid* grid,
                               uint32_t species_index, float mass_scale,
                               const float* outheights, size_t n_outheights, void* stream);
/* Cell index ((ix*ny)+iy)*nz+iz that fpg_grid_accumulate would use for each
 * slot [0, dispatch_count), 0xFFFFFFFF for inactive slots (the binning of
 * concentration_gridding.wgsl:332-336 on its own).  out_dev: device array. */
fpg_status fpg_grid_cell_indices(fpg_ctx* ctx, const fpg_particles* particles, const fpg_grid* grid,
                                 const float* outheights, size_t n_outheights, uint32_t* out_dev,
                                 void* stream);
/* The counts and raw scaled masses copied to host memory (page-locked for
 * overlap, e.g. fpg_host_alloc) on `stream` without waiting: the copy is
 * ordered after the grid's last accumulate, and the next accumulate into
 * this grid waits for it.  The host buffers are complete once `stream`
 * reaches this point (synchronize it, or make another stream wait on it).
 * Either pointer may be NULL. */
fpg_status fpg_grid_download_async(fpg_grid* grid, uint32_t* counts, uint32_t* mass_scaled, void* stream);
/* download_output (gridding.rs:191-219): counts, raw scaled masses and kg
 * (= scaled / mass_scale as f32); any pointer may be NULL. */
fpg_status fpg_grid_download(fpg_grid* g, uint32_t* counts, uint32_t* mass_scaled, float* mass_kg,
                             void* stream);
/* Device pointers of the count and scaled-mass grids (nx*ny*nz u32 each). */
uint32_t* fpg_grid_counts_device(fpg_grid* g);
uint32_t* fpg_grid_mass_device(fpg_grid* g);

/* ------------------------------------------------------------------------
 * Active-particle compaction (src/gpu/compaction.rs:447-505)
 * ---------------------------------------------------------------------- */
typedef struct fpg_compaction fpg_compaction;

fpg_status fpg_compaction_create(fpg_ctx* ctx, size_t capacity, fpg_compaction** out);
fpg_status fpg_compaction_destroy(fpg_compaction* c);
/* encode_compaction_with_reorder + download_active_count
 * (compaction.rs:447-505,290-302): a stable scan of the active bit over all
 * capacity slots; active slots move, in their original order, to
 * [0, active_count); every slot >= active_count receives its own previous
 * contents with the active bit cleared (compaction.wgsl:194-217).  Sets the
 * dispatch count to active_count (timeloop.rs:1254-1261).  `active_count`
 * (host, may be NULL) receives the count; `compacted_indices_dev` (optional
 * device array of capacity u32) receives the original slot of each
 * compacted position. */
fpg_status fpg_compact(fpg_ctx* ctx, fpg_particles* particles, fpg_compaction* c,
                       uint32_t* active_count, uint32_t* compacted_indices_dev, void* stream);

/* ------------------------------------------------------------------------
 * Spatial reorder by met cell (replaces the reference's optional host Morton
 * sort: ParticleStore::sort_spatially, src/particles/mod.rs:649-699, applied
 * by apply_spatial_sort_if_enabled, src/simulation/timeloop.rs:1414-1430)
 * ---------------------------------------------------------------------- */
typedef struct fpg_sorter fpg_sorter;

fpg_status fpg_sorter_create(fpg_ctx* ctx, size_t capacity, fpg_sorter** out);
fpg_status fpg_sorter_destroy(fpg_sorter* s);
/* Stable reorder of slots [0, dispatch_count) by the 3-D met cell of each
 * particle, key ((ix*ny)+iy)*nz+iz with ix = floor(clamp(cell_x+pos_x, 0,
 * nx-1)), iy likewise, iz = floor(clamp(level(pos_z), 0, nz-1)) and level()
 * the metres->level map of the advection (advection_dual_wind.wgsl:94-117);
 * inactive slots sort last, as the reference's INACTIVE_MORTON_KEY
 * (particles/mod.rs:27).  All fields move; slots >= dispatch_count keep
 * their place.  `perm_dev` (optional, dispatch_count u32) receives the old
 * slot of each new slot.  Philox streams follow the new slot, as they do
 * after the reference's own sort.  Field pointers change (the handle swaps
 * to the sorter's second block). */
fpg_status fpg_sort_by_cell(fpg_ctx* ctx, fpg_particles* particles, const fpg_met* met, fpg_sorter* sorter,
                            uint32_t* perm_dev, void* stream);

/* Largest slot count fpg_compaction_indices_static accepts (65536 tiles of
 * 2048 slots; its scratch is a 256 KiB static device array). */
#define FPG_STATIC_COMPACT_MAX_SLOTS (65536u * 2048u)

/* No counterpart in the reference.  The stable compaction scan of
 * fpg_compact for callers that cannot allocate device memory (their device
 * memory belongs to another allocator, or an allocation would stall a
 * latency-critical loop): it allocates nothing and keeps its per-tile
 * scratch in a static device array inside the library.  Inputs and outputs
 * are the caller's device buffers: `flags_dev` (n u32, bit 0 = active),
 * `indices_dev` (n u32; the first *active_count_dev entries receive the
 * original slot of each active particle, in slot order) and
 * `active_count_dev` (one u32).  Particle data is not moved.
 * n above FPG_STATIC_COMPACT_MAX_SLOTS returns FPG_ERR_VALUE_TOO_LARGE.
 * The first call for a device looks up the scratch array's device address
 * (once per device) and should come before any stream capture.  All calls
 * on a device share the one array: calls that overlap on the GPU race;
 * calls ordered on one stream are safe.  The looked-up address does not
 * survive a cudaDeviceReset of that device: do not call this entry point
 * again in a process after such a reset. */
fpg_status fpg_compaction_indices_static(fpg_ctx* ctx, const uint32_t* flags_dev, size_t n,
                                         uint32_t* indices_dev, uint32_t* active_count_dev,
                                         void* stream);

/* ------------------------------------------------------------------------
 * Philox utility (philox_rng.wgsl:441-464, src/gpu/rng.rs:198)
 * ---------------------------------------------------------------------- */
/* out_dev (device, 4*n floats): uniforms of blocks counter+0 .. counter+n-1. */
fpg_status fpg_philox_uniforms(fpg_ctx* ctx, const uint32_t key[2], const uint32_t counter[4],
                               size_t n_blocks, float* out_dev, uint32_t* out_raw_dev,
                               void* stream);

/* ------------------------------------------------------------------------
 * Convective boundary layer and convective mixing
 * ---------------------------------------------------------------------- */
/* HannaParams (src/pbl/mod.rs:23-57): 16 floats, 64 bytes per slot.
 * The record arrays below are read and written as 16-byte vectors: their
 * device pointers must be 16-byte aligned (INVALID_ARGUMENT otherwise). */
typedef struct fpg_hanna_params {
    float ust, wst, ol, h, zeta, sigu, sigv, sigw, dsigwdz, dsigw2dz, tlu, tlv, tlw;
    float pad[3];
} fpg_hanna_params;

/* CblSamplingInput (src/gpu/cbl.rs:38-50): uniforms in [0, 1). */
typedef struct fpg_cbl_sampling_input {
    float branch_uniform, gaussian_uniform0, gaussian_uniform1, pad0;
} fpg_cbl_sampling_input;

/* CblSamplingOutput (src/gpu/cbl.rs:66-92). */
typedef struct fpg_cbl_sampling_output {
    float sampled_w_m_s;
    float updraft_weight, updraft_mean_m_s, updraft_sigma_m_s;
    float downdraft_weight, downdraft_mean_m_s, downdraft_sigma_m_s;
    float second_moment_w2, third_moment_w3, skewness, transition, z_over_h;
} fpg_cbl_sampling_output;

/* dispatch_hanna_params_gpu (src/gpu/hanna.rs:238-330, hanna_params.wgsl:
 * 231-258): for each slot [0, dispatch_count) the PBL cell at
 * floor(clamp(cell + pos)), 1/L -> L (hanna.rs:169-174) and
 * compute_hanna_params (physics/hanna.rs:49-163); inactive slots get an
 * all-zero record.  out_dev: device array of n_out records.  Errors:
 * LengthMismatch (n_out != dispatch_count), ZeroPblShape, NotReady. */
fpg_status fpg_dispatch_hanna_params(fpg_ctx* ctx, const fpg_particles* particles, const fpg_pbl* pbl,
                                     fpg_hanna_params* out_dev, size_t n_out, void* stream);

/* encode_update_particles_turbulence_langevin_gpu_with_hanna_buffer_and_kernel
 * (src/gpu/langevin.rs:248-329, langevin.wgsl:307-424): the turbulence update
 * of every active slot [0, dispatch_count) from its HannaParams record — the
 * separated Hanna -> Langevin path of the reference's validation and backward
 * loops — with the Philox block layout of fpg_langevin_fused; records from
 * fpg_dispatch_hanna_params give the fused kernel's results bit for bit.
 * Sigma and T_L pass through sanitize_positive and a zero T_L gives zero
 * turbulence (langevin.wgsl:189-238).  next_counter = base + n * blocks per
 * slot (1 for n_substeps <= 2, else 2).  Errors: MismatchedInputLengths
 * (n_hanna != dispatch_count -> LENGTH_MISMATCH), InvalidTimeStep. */
fpg_status fpg_langevin_with_hanna(fpg_ctx* ctx, fpg_particles* particles, const fpg_hanna_params* hanna_dev,
                                   size_t n_hanna, float dt, float rho_grad_over_rho, uint32_t n_substeps,
                                   float min_height_m, const uint32_t key[2], const uint32_t base_counter[4],
                                   uint32_t next_counter[4], void* stream);

/* sample_cbl_vertical_velocity_gpu (src/gpu/cbl.rs:204-319, cbl.wgsl:251-298):
 * per slot [0, dispatch_count) the CBL bi-Gaussian PDF of w' from the slot's
 * height and Hanna record (h, w*, sigma_w, L; physics/cbl.rs:126-226) and one
 * sample (physics/cbl.rs:274-288); inactive slots get an all-zero output.
 * hanna_dev, inputs_dev, out_dev: device arrays.  Errors:
 * MismatchedInputLengths (n_hanna or n_inputs != dispatch_count). */
fpg_status fpg_cbl_sample(fpg_ctx* ctx, const fpg_particles* particles, const fpg_hanna_params* hanna_dev,
                          size_t n_hanna, const fpg_cbl_sampling_input* inputs_dev, size_t n_inputs,
                          fpg_cbl_sampling_output* out_dev, void* stream);

/* The same sample with its inputs formed on the device: sigma_w of the Hanna
 * parameters at the slot's PBL cell, and the first three uniforms of the
 * Philox block at counter + slot (sample_cbl_vertical_velocity_with_rng,
 * physics/cbl.rs:291-295, on a stream that starts at that counter).
 * Errors: ZeroPblShape, NotReady. */
fpg_status fpg_cbl_sample_philox(fpg_ctx* ctx, const fpg_particles* particles, const fpg_pbl* pbl,
                                 const uint32_t key[2], const uint32_t counter[4],
                                 fpg_cbl_sampling_output* out_dev, void* stream);

/* SimplifiedEmanuelInputs (physics/convection.rs:68-82). */
typedef struct fpg_convection_inputs {
    const float* level_interfaces_m;        /* n_levels + 1 interfaces [m] */
    size_t n_interfaces;
    float convective_precip_mm_h;
    float convective_velocity_scale_m_s;
    float boundary_layer_height_m;
    int32_t has_cape_override;              /* Option<f32>: 0 = None */
    float cape_override_j_kg;
} fpg_convection_inputs;

/* The scalars of SimplifiedEmanuelColumn (physics/convection.rs:111-133) and
 * the matrix's mixing fraction (physics/convection.rs:143-154). */
typedef struct fpg_convection_column {
    int32_t is_active;
    float cape_j_kg;
    uint32_t cloud_base_level;
    uint32_t cloud_top_level;
    float convective_timescale_s;
    float mixing_fraction;
} fpg_convection_column;

/* build_simplified_convection_chain (physics/convection.rs:462-467) on the
 * host: the column diagnostics and the column-major L*L redistribution
 * matrix (L = n_interfaces - 1).  centers_out, mass_flux_out and
 * detrainment_out (L floats each) may be NULL.  Errors: TooFewLevels,
 * NonMonotonicInterfaces, InvalidBoundaryLayerHeight, InvalidTimeStep,
 * NonStochasticColumn. */
fpg_status fpg_convection_build_chain(const fpg_convection_inputs* inputs, float dt_seconds,
                                      fpg_convection_column* column, float* matrix_out, float* centers_out,
                                      float* mass_flux_out, float* detrainment_out);
/* level_index_from_height (physics/convection.rs:469-489). */
size_t fpg_convection_level_index(const float* level_interfaces_m, size_t n_interfaces, float height_m);
/* apply_redistribution_matrix (physics/convection.rs:370-392) on the host:
 * destination = M * source.  Errors: ProfileLengthMismatch. */
fpg_status fpg_convection_apply_profile(const float* matrix_column_major, size_t level_count,
                                        const float* source, size_t n_source, float* destination);

/* A convective redistribution matrix on the device
 * (ConvectiveRedistributionMatrix, physics/convection.rs:143-219).
 * Errors of create: InvalidLevelCount (0 -> ZERO_SHAPE, > 65535 ->
 * VALUE_TOO_LARGE). */
typedef struct fpg_convection fpg_convection;
fpg_status fpg_convection_create(fpg_ctx* ctx, size_t level_count, fpg_convection** out);
fpg_status fpg_convection_destroy(fpg_convection* conv);
/* Host arrays: the column-major matrix (source * L + destination, L*L
 * floats) and the L+1 level interfaces [m].  Validates the columns as the
 * reference's matrix type does (entries >= -1e-4 and finite, column sums
 * within 1e-4 of 1), uploads both, and forms the expected destination height
 * of every source level (physics/convection.rs:398-427) on the device.
 * Returns after the upload.  Errors: LENGTH_MISMATCH (MatrixLengthMismatch /
 * InvalidLevelInterfaces), NON_STOCHASTIC_COLUMN. */
fpg_status fpg_convection_set_matrix(fpg_convection* conv, const float* matrix_column_major, size_t n_matrix,
                                     const float* level_interfaces_m, size_t n_interfaces, void* stream);
/* The expected destination heights (L floats, clamped to the column). */
fpg_status fpg_convection_heights(const fpg_convection* conv, float* heights_host);
/* dispatch_convective_mixing_gpu (src/gpu/convection.rs:71-250,
 * convective_mixing.wgsl:75-113): each active slot [0, dispatch_count) moves
 * to the expected destination height of its source level and records that
 * level in `cbt`. */
fpg_status fpg_convective_mixing(fpg_ctx* ctx, fpg_particles* particles, const fpg_convection* conv,
                                 void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FPG_H */
