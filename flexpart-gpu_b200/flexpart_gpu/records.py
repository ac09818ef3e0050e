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
