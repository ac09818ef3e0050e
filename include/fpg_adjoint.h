/*
 * fpg_adjoint.h — source inversion: a forward/backward pair over the batched
 * step (fpg_driver.h), in the role a differentiable operator plays in an
 * autodiff framework.
 *
 * No counterpart in the reference, which has no adjoint, autodiff or finite
 * differences (its "backward" time loop, simulation/timeloop.rs:1433-1448,
 * is FLEXPART's time-reversed receptor mode, not a gradient).
 *
 * forward: runs the production step (fpg_step's physics: dual-time
 *   trilinear advection, Hanna + Langevin with sub-steps and reflection,
 *   dry and wet decay) for every source from the start time to the end time
 *   and returns, per receptor, the time-integrated smooth concentration
 *       sim_r = sum over sampling steps, over particles p of the receptor's
 *               instance, of m_p * W_r(x_p, y_p, z_p)
 *   where W_r is the cloud-in-cell weight of receptor cell (i, j)
 *   (tent functions of width one cell centred on the cell centre, in grid
 *   coordinates) times a vertical weight that is 1 below
 *   receptor_top_m - ramp/2, 0 above receptor_top_m + ramp/2 and linear
 *   between.  Particle state is checkpointed every K steps, or the tape of
 *   every step is recorded during the forward itself (K = 0).
 * backward: given dL/dsim_r, returns dL/d(source mass), dL/d(source
 *   position: lon, lat, z of the release box, moved rigidly) and dL/d(wind
 *   bias) for a bias field b added to u, v, w at every met node of every
 *   frame.  Each K-step window is recomputed from its checkpoint while a
 *   tape of the per-step local derivatives is recorded, then reversed step
 *   by step.  The Philox noise is the forward's (same counters), so the
 *   gradient is that of the forward map under fixed random numbers.
 *
 * Derivatives follow the computed path: the PBL and wet-scavenging cell a
 * particle falls in, the dry-deposition height test and the Hanna regime are
 * piecewise constant in position (zero derivative); clamps pass the
 * derivative only strictly inside their range; reflection flips the sign of
 * the height and vertical-velocity tangents.
 */
#ifndef FPG_ADJOINT_H
#define FPG_ADJOINT_H

#include "fpg_driver.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A receptor: cell (i, j) of the met grid's horizontal plane, observed in the
 * lowest layer, belonging to one inversion instance. */
typedef struct fpg_receptor {
    uint32_t instance;
    uint32_t i, j;
} fpg_receptor;

typedef struct fpg_inverse_config {
    fpg_batch_config batch;          /* clock, met ring, physics, release grid; its out_* grid and
                                        output_every_steps are not used */
    uint32_t sample_every_steps;     /* receptors sampled after steps k with (k + 1) % every == 0 */
    float receptor_top_m;            /* top of the observed layer (100 m) */
    float receptor_ramp_m;           /* width of the vertical weight's linear ramp (> 0) */
    uint32_t checkpoint_every;       /* K >= 1: particle state saved every K steps and each K-step
                                        window recomputed with its tape in the backward (memory:
                                        steps/K checkpoints of 44 B per slot + K x 80 B per slot);
                                        0: the forward records the tape of every step (no recompute;
                                        steps x 80 B per slot) */
    uint32_t tape_tail_windows;      /* with K >= 1: the forward also records the tape of its last
                                        W windows (W x K x 80 B per slot, replacing their
                                        checkpoints), which the backward reverses without
                                        recomputing them; 0 = every window recomputed */
} fpg_inverse_config;

typedef struct fpg_inverse fpg_inverse;

/* Sources are scenarios of a batch (own release, key and counter);
 * source_instance[s] < n_instances groups them into independent inversion
 * instances (NULL: all in instance 0).  Receptors of instance n see only
 * that instance's particles. */
fpg_status fpg_inverse_create(fpg_ctx* ctx, const fpg_inverse_config* cfg, const fpg_batch_scenario* sources,
                              const uint32_t* source_instance, size_t n_sources, size_t met_nx, size_t met_ny,
                              size_t met_nz, const float* level_heights, const fpg_receptor* receptors,
                              size_t n_receptors, fpg_inverse** out);
fpg_status fpg_inverse_destroy(fpg_inverse* inv);
/* Frame k of the met ring, as fpg_batch_upload_frame. */
fpg_status fpg_inverse_upload_frame(fpg_inverse* inv, uint32_t k, const float* u, const float* v, const float* w,
                                    const fpg_surface_cell* surface, const float* precipitation_mm_h);
/* Source parameters: total mass [kg] per source and the release box's lower
 * corner (lon_min, lat_min, z_min) per source (3 doubles; the box keeps its
 * extent).  Either may be NULL (unchanged). */
fpg_status fpg_inverse_set_sources(fpg_inverse* inv, const double* mass_kg, const double* position);
/* Wind bias: nx*ny*nz*3 floats, node ((ix*ny)+iy)*nz+iz then (u, v, w);
 * NULL sets it to zero. */
fpg_status fpg_inverse_set_wind_bias(fpg_inverse* inv, const float* bias);
/* Runs the whole forward run and writes sim_r (n_receptors doubles). */
fpg_status fpg_inverse_forward(fpg_inverse* inv, double* simulated);
/* After fpg_inverse_forward with the same parameters (and, with K >= 1, once
 * per forward: the recompute consumes the checkpointed state): the gradient of a
 * loss L given dL/dsim_r.  d_mass (n_sources), d_position (n_sources * 3:
 * d/dlon [per degree], d/dlat, d/dz [per metre]) and d_wind_bias (nodes*3)
 * may each be NULL. */
fpg_status fpg_inverse_backward(fpg_inverse* inv, const double* d_simulated, double* d_mass, double* d_position,
                                float* d_wind_bias);
/* The batch the inversion runs on (launch-shape tuning, particles). */
fpg_batch* fpg_inverse_batch(fpg_inverse* inv);
/* Device bytes held for checkpoints, tape and adjoint state. */
uint64_t fpg_inverse_device_bytes(const fpg_inverse* inv);

#ifdef __cplusplus
}
#endif

#endif /* FPG_ADJOINT_H */
