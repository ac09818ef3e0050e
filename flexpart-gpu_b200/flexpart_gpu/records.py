"""Exchange records of the C ABI (include/fpg.h) as numpy dtypes and ctypes
structures.

The particle record is byte-compatible with the reference's 96-byte
``#[repr(C)] Particle`` (src/particles/mod.rs:76-168); the surface record
with ``SurfaceCellInputGpu`` (src/gpu/pbl.rs:35-50).
"""
from __future__ import annotations

import ctypes

import numpy as np

MAX_SPECIES = 4
FLAG_ACTIVE = 1
MAX_LEVELS = 256

PARTICLE_DTYPE = np.dtype(
    [
        ("pos_x", "<f4"), ("pos_y", "<f4"), ("pos_z", "<f4"),
        ("cell_x", "<i4"), ("cell_y", "<i4"), ("flags", "<u4"),
        ("mass", "<f4", (MAX_SPECIES,)),
        ("vel_u", "<f4"), ("vel_v", "<f4"), ("vel_w", "<f4"),
        ("turb_u", "<f4"), ("turb_v", "<f4"), ("turb_w", "<f4"),
        ("time", "<i4"), ("timestep", "<i4"), ("time_mem", "<i4"), ("time_split", "<i4"),
        ("release_point", "<i4"), ("class_id", "<i4"), ("cbt", "<i4"), ("pad0", "<u4"),
    ]
)
assert PARTICLE_DTYPE.itemsize == 96

# HannaParams (src/pbl/mod.rs:23-57), fpg_hanna_params: 64 bytes per slot.
HANNA_PARAMS_DTYPE = np.dtype([(n, "<f4") for n in (
    "ust", "wst", "ol", "h", "zeta", "sigu", "sigv", "sigw", "dsigwdz", "dsigw2dz", "tlu", "tlv", "tlw")]
    + [("pad", "<f4", (3,))])
assert HANNA_PARAMS_DTYPE.itemsize == 64

# CblSamplingInput / CblSamplingOutput (src/gpu/cbl.rs:38-92).
CBL_INPUT_DTYPE = np.dtype([("branch_uniform", "<f4"), ("gaussian_uniform0", "<f4"),
                            ("gaussian_uniform1", "<f4"), ("pad0", "<f4")])
CBL_OUTPUT_DTYPE = np.dtype([(n, "<f4") for n in (
    "sampled_w_m_s", "updraft_weight", "updraft_mean_m_s", "updraft_sigma_m_s", "downdraft_weight",
    "downdraft_mean_m_s", "downdraft_sigma_m_s", "second_moment_w2", "third_moment_w3", "skewness",
    "transition", "z_over_h")])
assert CBL_INPUT_DTYPE.itemsize == 16 and CBL_OUTPUT_DTYPE.itemsize == 48

SURFACE_DTYPE = np.dtype(
    [
        ("surface_pressure_pa", "<f4"), ("temperature_2m_k", "<f4"),
        ("u10_ms", "<f4"), ("v10_ms", "<f4"),
        ("surface_stress_n_m2", "<f4"), ("sensible_heat_flux_w_m2", "<f4"),
        ("solar_radiation_w_m2", "<f4"), ("mixing_height_m", "<f4"),
        ("friction_velocity_ms", "<f4"), ("inv_obukhov_length_per_m", "<f4"),
        ("pad0", "<f4"), ("pad1", "<f4"),
    ]
)
assert SURFACE_DTYPE.itemsize == 48

# Structure-of-arrays field ids (FPG_FIELD_* in include/fpg.h) and dtypes.
FIELDS = [
    ("pos_x", np.float32), ("pos_y", np.float32), ("pos_z", np.float32),
    ("cell_x", np.int32), ("cell_y", np.int32), ("flags", np.uint32),
    ("mass0", np.float32), ("mass1", np.float32), ("mass2", np.float32), ("mass3", np.float32),
    ("vel_u", np.float32), ("vel_v", np.float32), ("vel_w", np.float32),
    ("turb_u", np.float32), ("turb_v", np.float32), ("turb_w", np.float32),
    ("time", np.int32), ("timestep", np.int32), ("time_mem", np.int32), ("time_split", np.int32),
    ("release_point", np.int32), ("class_id", np.int32), ("cbt", np.int32),
]
FIELD_ID = {name: i for i, (name, _) in enumerate(FIELDS)}
FIELD_DTYPE = {name: dt for name, dt in FIELDS}

# Forcing modes and stage bits (include/fpg.h).
FORCING_NONE, FORCING_UNIFORM, FORCING_PER_PARTICLE, FORCING_PER_CELL = 0, 1, 2, 3
STAGE_ADVECT, STAGE_TURBULENCE, STAGE_DRY, STAGE_WET = 1, 2, 4, 8
STAGE_ALL = 15


class StepParams(ctypes.Structure):
    """``fpg_step_params`` (include/fpg.h)."""

    _fields_ = [
        ("stages", ctypes.c_uint32),
        ("alpha", ctypes.c_float),
        ("dt_seconds", ctypes.c_float),
        ("turb_dt_seconds", ctypes.c_float),
        ("x_grid_per_meter", ctypes.c_float),
        ("y_grid_per_meter", ctypes.c_float),
        ("z_grid_per_meter", ctypes.c_float),
        ("n_substeps", ctypes.c_uint32),
        ("min_height_m", ctypes.c_float),
        ("rho_grad_over_rho", ctypes.c_float),
        ("key", ctypes.c_uint32 * 2),
        ("counter", ctypes.c_uint32 * 4),
        ("dry_reference_height_m", ctypes.c_float),
        ("dry_mode", ctypes.c_int32),
        ("dry_velocity_m_s", ctypes.c_float),
        ("dry_velocity_dev", ctypes.c_void_p),
        ("dry_probability_dev", ctypes.c_void_p),
        ("wet_mode", ctypes.c_int32),
        ("wet_lambda_s_inv", ctypes.c_float),
        ("wet_fraction", ctypes.c_float),
        ("wet_lambda_dev", ctypes.c_void_p),
        ("wet_fraction_dev", ctypes.c_void_p),
        ("wet_cells", ctypes.c_void_p),
        ("wet_probability_dev", ctypes.c_void_p),
    ]

    @classmethod
    def production(cls, **kw) -> "StepParams":
        """The forward loop's production settings
        (src/simulation/timeloop.rs:1062-1113): all stages, 4 vertical
        sub-steps, 0.01 m reflection floor, 15 m dry reference height."""
        p = cls()
        p.stages = STAGE_ALL
        p.alpha = 0.0
        p.dt_seconds = 900.0
        p.turb_dt_seconds = 900.0
        p.x_grid_per_meter = 1.0
        p.y_grid_per_meter = 1.0
        p.z_grid_per_meter = 1.0
        p.n_substeps = 4
        p.min_height_m = 0.01
        p.rho_grad_over_rho = 0.0
        p.dry_reference_height_m = 15.0
        p.dry_mode = FORCING_NONE
        p.wet_mode = FORCING_NONE
        for k, v in kw.items():
            if k in ("key", "counter"):
                arr = getattr(p, k)
                for i, x in enumerate(v):
                    arr[i] = int(x) & 0xFFFFFFFF
            else:
                setattr(p, k, v)
        return p


class PblOptions(ctypes.Structure):
    """``fpg_pbl_options``: PblComputationOptions (src/io/pbl_params.rs:35-68)."""

    _fields_ = [
        ("roughness_length_m", ctypes.c_float),
        ("wind_reference_height_m", ctypes.c_float),
        ("heat_flux_neutral_threshold_w_m2", ctypes.c_float),
        ("fallback_mixing_height_m", ctypes.c_float),
        ("hmix_min_m", ctypes.c_float),
        ("hmix_max_m", ctypes.c_float),
    ]

    @classmethod
    def default(cls) -> "PblOptions":
        return cls(0.1, 10.0, 1.0, 800.0, 100.0, 4500.0)


class Release(ctypes.Structure):
    """``fpg_release`` (include/fpg_driver.h): ReleaseConfig as the release
    manager reads it (src/release/mod.rs:199-254)."""

    _fields_ = [
        ("start_seconds", ctypes.c_int64), ("end_seconds", ctypes.c_int64),
        ("lon_min", ctypes.c_double), ("lon_max", ctypes.c_double),
        ("lat_min", ctypes.c_double), ("lat_max", ctypes.c_double),
        ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
        ("mass_kg", ctypes.c_double), ("particle_count", ctypes.c_uint64),
    ]


class GridDomain(ctypes.Structure):
    """``fpg_grid_domain``: GridDomain (src/coords/mod.rs)."""

    _fields_ = [("xlon0", ctypes.c_double), ("ylat0", ctypes.c_double), ("dx", ctypes.c_double),
                ("dy", ctypes.c_double), ("nx", ctypes.c_uint64), ("ny", ctypes.c_uint64)]


class ForwardConfig(ctypes.Structure):
    """``fpg_forward_config``: ForwardTimeLoopConfig (timeloop.rs:67-124)."""

    _fields_ = [
        ("start_seconds", ctypes.c_int64), ("end_seconds", ctypes.c_int64), ("timestep_seconds", ctypes.c_int64),
        ("clamp_time_bounds", ctypes.c_int32),
        ("x_grid_per_meter", ctypes.c_float), ("y_grid_per_meter", ctypes.c_float),
        ("z_grid_per_meter", ctypes.c_float),
        ("pbl_options", PblOptions),
        ("dry_reference_height_m", ctypes.c_float),
        ("philox_key", ctypes.c_uint32 * 2), ("initial_philox_counter", ctypes.c_uint32 * 4),
        ("sort_interval_steps", ctypes.c_uint32), ("use_compaction", ctypes.c_int32),
        ("n_substeps", ctypes.c_uint32), ("min_height_m", ctypes.c_float),
    ]


class BatchScenario(ctypes.Structure):
    """``fpg_batch_scenario``: one release with its own Philox key and
    initial counter (include/fpg_driver.h)."""

    _fields_ = [("release", Release), ("key", ctypes.c_uint32 * 2), ("counter", ctypes.c_uint32 * 4)]


class BatchConfig(ctypes.Structure):
    """``fpg_batch_config``: the shared clock, met ring, physics options and
    per-scenario output grid of a batched ensemble."""

    _fields_ = [
        ("start_seconds", ctypes.c_int64), ("end_seconds", ctypes.c_int64), ("timestep_seconds", ctypes.c_int64),
        ("frame_seconds", ctypes.c_int64), ("n_frames", ctypes.c_uint32),
        ("x_grid_per_meter", ctypes.c_float), ("y_grid_per_meter", ctypes.c_float),
        ("z_grid_per_meter", ctypes.c_float),
        ("pbl_options", PblOptions),
        ("dry_reference_height_m", ctypes.c_float), ("dry_velocity_m_s", ctypes.c_float),
        ("rho_grad_over_rho", ctypes.c_float), ("n_substeps", ctypes.c_uint32), ("min_height_m", ctypes.c_float),
        ("wet_from_precipitation", ctypes.c_int32), ("wet_gas_a", ctypes.c_float), ("wet_gas_b", ctypes.c_float),
        ("release_grid", GridDomain),
        ("out_nx", ctypes.c_uint32), ("out_ny", ctypes.c_uint32), ("out_nz", ctypes.c_uint32),
        ("outheights", ctypes.c_void_p), ("output_every_steps", ctypes.c_uint32),
    ]


class BatchTuning(ctypes.Structure):
    """``fpg_batch_tuning``: launch shape of the batched particle pass."""

    _fields_ = [("block_threads", ctypes.c_uint32), ("min_blocks_per_sm", ctypes.c_uint32),
                ("particles_per_thread", ctypes.c_uint32), ("step_ms", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Receptor(ctypes.Structure):
    """``fpg_receptor`` (include/fpg_adjoint.h)."""

    _fields_ = [("instance", ctypes.c_uint32), ("i", ctypes.c_uint32), ("j", ctypes.c_uint32)]


class InverseConfig(ctypes.Structure):
    """``fpg_inverse_config`` (include/fpg_adjoint.h)."""

    _fields_ = [("batch", BatchConfig), ("sample_every_steps", ctypes.c_uint32),
                ("receptor_top_m", ctypes.c_float), ("receptor_ramp_m", ctypes.c_float),
                ("checkpoint_every", ctypes.c_uint32), ("tape_tail_windows", ctypes.c_uint32)]


class ReceptorRelease(ctypes.Structure):
    """``fpg_receptor_release``: BackwardReceptorConfig (timeloop.rs:150-163)."""

    _fields_ = [("lon", ctypes.c_double), ("lat", ctypes.c_double), ("z_m", ctypes.c_double),
                ("particle_count", ctypes.c_uint64), ("mass_kg", ctypes.c_double)]


class SourceRegion(ctypes.Structure):
    """``fpg_source_region``: BackwardSourceRegionConfig (timeloop.rs:170-197)."""

    _fields_ = [("lon_min", ctypes.c_double), ("lon_max", ctypes.c_double), ("lat_min", ctypes.c_double),
                ("lat_max", ctypes.c_double), ("z_min_m", ctypes.c_double), ("z_max_m", ctypes.c_double)]


class SourceCollection(ctypes.Structure):
    """``fpg_source_collection``: BackwardSourceCollection (timeloop.rs:201-206)."""

    _fields_ = [("hit_count", ctypes.c_uint64), ("total_mass_kg", ctypes.c_float), ("pad", ctypes.c_float),
                ("total_mass_kg_f64", ctypes.c_double)]


class BackwardConfig(ctypes.Structure):
    """``fpg_backward_config``: BackwardTimeLoopConfig (timeloop.rs:226-251)."""

    _fields_ = [
        ("start_seconds", ctypes.c_int64), ("end_seconds", ctypes.c_int64), ("timestep_seconds", ctypes.c_int64),
        ("clamp_time_bounds", ctypes.c_int32),
        ("x_grid_per_meter", ctypes.c_float), ("y_grid_per_meter", ctypes.c_float),
        ("z_grid_per_meter", ctypes.c_float),
        ("pbl_options", PblOptions),
        ("dry_reference_height_m", ctypes.c_float),
        ("philox_key", ctypes.c_uint32 * 2), ("initial_philox_counter", ctypes.c_uint32 * 4),
        ("n_substeps", ctypes.c_uint32), ("min_height_m", ctypes.c_float),
    ]


class MetBracket(ctypes.Structure):
    """``fpg_met_bracket``: MetTimeBracket (timeloop.rs:270-285)."""

    _fields_ = [
        ("wind_t0_u", ctypes.c_void_p), ("wind_t0_v", ctypes.c_void_p), ("wind_t0_w", ctypes.c_void_p),
        ("wind_t1_u", ctypes.c_void_p), ("wind_t1_v", ctypes.c_void_p), ("wind_t1_w", ctypes.c_void_p),
        ("surface_t0", ctypes.c_void_p), ("surface_t1", ctypes.c_void_p),
        ("time_t0_seconds", ctypes.c_int64), ("time_t1_seconds", ctypes.c_int64),
    ]


class Forcing(ctypes.Structure):
    """``fpg_forcing``: ForwardStepForcing (timeloop.rs:347-358)."""

    _fields_ = [
        ("dry_mode", ctypes.c_int32), ("dry_velocity_m_s", ctypes.c_float),
        ("dry_velocity_per_slot", ctypes.c_void_p),
        ("wet_mode", ctypes.c_int32), ("wet_lambda_s_inv", ctypes.c_float), ("wet_fraction", ctypes.c_float),
        ("wet_lambda_per_slot", ctypes.c_void_p), ("wet_fraction_per_slot", ctypes.c_void_p),
        ("wet_cells", ctypes.c_void_p),
        ("rho_grad_over_rho", ctypes.c_float),
    ]


class StepReport(ctypes.Structure):
    """``fpg_step_report``: ForwardStepReport (timeloop.rs:1294-1308)."""

    _fields_ = [
        ("step_index", ctypes.c_uint64), ("simulation_time_seconds", ctypes.c_int64),
        ("interpolation_alpha", ctypes.c_float), ("released_count", ctypes.c_uint64),
        ("first_released_slot", ctypes.c_uint64), ("active_particle_count", ctypes.c_uint64),
        ("next_philox_counter", ctypes.c_uint32 * 4),
    ]


class StepTiming(ctypes.Structure):
    """``fpg_step_timing``: the per-section timing of one forward step, the
    device form of StepTimingReport (timeloop.rs:398-467), in ms."""

    _fields_ = [
        ("step_index", ctypes.c_uint64), ("sort_ms", ctypes.c_double), ("release_ms", ctypes.c_double),
        ("met_bracket_ms", ctypes.c_double), ("pbl_ms", ctypes.c_double), ("step_ms", ctypes.c_double),
        ("compaction_ms", ctypes.c_double), ("gpu_total_ms", ctypes.c_double),
        ("host_call_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
    ]


class ConvectionInputs(ctypes.Structure):
    """fpg_convection_inputs: SimplifiedEmanuelInputs (physics/convection.rs:68-82)."""
    _fields_ = [
        ("level_interfaces_m", ctypes.c_void_p), ("n_interfaces", ctypes.c_size_t),
        ("convective_precip_mm_h", ctypes.c_float), ("convective_velocity_scale_m_s", ctypes.c_float),
        ("boundary_layer_height_m", ctypes.c_float), ("has_cape_override", ctypes.c_int32),
        ("cape_override_j_kg", ctypes.c_float),
    ]


class ConvectionColumn(ctypes.Structure):
    """fpg_convection_column: the scalars of SimplifiedEmanuelColumn plus the
    matrix's mixing fraction (physics/convection.rs:111-154)."""
    _fields_ = [
        ("is_active", ctypes.c_int32), ("cape_j_kg", ctypes.c_float), ("cloud_base_level", ctypes.c_uint32),
        ("cloud_top_level", ctypes.c_uint32), ("convective_timescale_s", ctypes.c_float),
        ("mixing_fraction", ctypes.c_float),
    ]


def particles_from_soa(fields: dict, n: int) -> np.ndarray:
    """Builds fpg_particle records from a dict of per-field arrays."""
    rec = np.zeros(n, dtype=PARTICLE_DTYPE)
    for name, arr in fields.items():
        if name.startswith("mass") and name != "mass":
            rec["mass"][:, int(name[4:])] = arr
        elif name == "mass":
            rec["mass"][:] = arr
        else:
            rec[name] = arr
    return rec


def soa_from_particles(rec: np.ndarray) -> dict:
    """Splits fpg_particle records into per-field arrays (FIELDS names)."""
    out = {}
    for name, dt in FIELDS:
        if name.startswith("mass"):
            out[name] = np.ascontiguousarray(rec["mass"][:, int(name[4:])]).astype(dt)
        else:
            out[name] = np.ascontiguousarray(rec[name]).astype(dt)
    return out
