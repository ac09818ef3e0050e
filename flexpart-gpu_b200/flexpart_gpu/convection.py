"""Convective mixing: the simplified Emanuel column, its redistribution
matrix, and the matrix applied to particle heights on the device.

Mirrors physics/convection.rs (the column and matrix, built on the host as
the reference builds them, here by the library's C++ host code) and
src/gpu/convection.rs (dispatch_convective_mixing_gpu).  The device object
``ConvectiveMixing`` holds one matrix: setting it validates the columns,
uploads it, and forms the expected destination height of every source level
once; each dispatch then moves every active slot to the height of its
source level and records that level in ``cbt``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._lib import FpgError, check, lib
from .api import Context, Particles, _p, _vp
from .records import ConvectionColumn, ConvectionInputs

__all__ = [
    "SimplifiedEmanuelInputs", "SimplifiedEmanuelColumn", "ConvectiveRedistributionMatrix",
    "build_simplified_convection_chain", "level_index_from_height", "apply_redistribution_matrix",
    "ConvectiveMixing", "dispatch_convective_mixing_gpu",
]


@dataclass
class SimplifiedEmanuelInputs:
    """physics/convection.rs:68-82."""
    level_interfaces_m: list
    convective_precip_mm_h: float
    convective_velocity_scale_m_s: float
    boundary_layer_height_m: float
    cape_override_j_kg: float | None = None


@dataclass
class SimplifiedEmanuelColumn:
    """physics/convection.rs:111-133."""
    level_interfaces_m: np.ndarray
    level_centers_m: np.ndarray
    is_active: bool
    cape_j_kg: float
    cloud_base_level: int
    cloud_top_level: int
    mass_flux_profile_kg_m2_s: np.ndarray
    detrainment_weights: np.ndarray
    convective_timescale_s: float

    def level_count(self) -> int:
        return self.level_centers_m.size


@dataclass
class ConvectiveRedistributionMatrix:
    """physics/convection.rs:143-219: coefficients_column_major[source *
    L + destination]."""
    coefficients_column_major: np.ndarray
    mixing_fraction: float = 0.0
    cloud_base_level: int = 0
    cloud_top_level: int = 0
    _level_count: int = field(default=0, repr=False)

    def level_count(self) -> int:
        return self._level_count

    def coefficient(self, destination_level: int, source_level: int) -> float:
        return float(self.coefficients_column_major[source_level * self._level_count + destination_level])


def build_simplified_convection_chain(inputs: SimplifiedEmanuelInputs, dt_seconds: float):
    """(column, matrix) of build_simplified_convection_chain
    (physics/convection.rs:462-467)."""
    iface = np.ascontiguousarray(inputs.level_interfaces_m, np.float32)
    n = max(iface.size - 1, 0)
    c_in = ConvectionInputs()
    c_in.level_interfaces_m = iface.ctypes.data if iface.size else None
    c_in.n_interfaces = iface.size
    c_in.convective_precip_mm_h = inputs.convective_precip_mm_h
    c_in.convective_velocity_scale_m_s = inputs.convective_velocity_scale_m_s
    c_in.boundary_layer_height_m = inputs.boundary_layer_height_m
    c_in.has_cape_override = 0 if inputs.cape_override_j_kg is None else 1
    c_in.cape_override_j_kg = 0.0 if inputs.cape_override_j_kg is None else inputs.cape_override_j_kg
    col = ConvectionColumn()
    m = np.zeros(max(n * n, 1), np.float32)
    centers = np.zeros(max(n, 1), np.float32)
    flux = np.zeros(max(n, 1), np.float32)
    det = np.zeros(max(n, 1), np.float32)
    check(lib.fpg_convection_build_chain(ctypes.byref(c_in), dt_seconds, ctypes.byref(col), _p(m), _p(centers),
                                         _p(flux), _p(det)), "fpg_convection_build_chain")
    column = SimplifiedEmanuelColumn(iface.copy(), centers[:n].copy(), bool(col.is_active), col.cape_j_kg,
                                     int(col.cloud_base_level), int(col.cloud_top_level), flux[:n].copy(),
                                     det[:n].copy(), col.convective_timescale_s)
    if col.is_active:
        base, top = int(col.cloud_base_level), int(col.cloud_top_level)
    else:
        base, top = 0, max(n - 1, 0)       # from_column_major defaults (physics/convection.rs:174-180)
    matrix = ConvectiveRedistributionMatrix(m[:n * n].copy(), col.mixing_fraction, base, top, n)
    return column, matrix


def level_index_from_height(level_interfaces_m, height_m: float) -> int:
    """physics/convection.rs:469-489."""
    iface = np.ascontiguousarray(level_interfaces_m, np.float32)
    return int(lib.fpg_convection_level_index(_p(iface) if iface.size else None, iface.size, height_m))


def apply_redistribution_matrix(matrix: ConvectiveRedistributionMatrix, source_profile) -> np.ndarray:
    """destination = M * source (physics/convection.rs:370-392)."""
    src = np.ascontiguousarray(source_profile, np.float32)
    dst = np.zeros(max(matrix.level_count(), 1), np.float32)
    check(lib.fpg_convection_apply_profile(_p(matrix.coefficients_column_major), matrix.level_count(), _p(src),
                                           src.size, _p(dst)), "fpg_convection_apply_profile")
    return dst[:matrix.level_count()]


class ConvectiveMixing:
    """A redistribution matrix resident on the device (fpg_convection)."""

    def __init__(self, ctx: Context, level_count: int):
        self.ctx, self.level_count = ctx, level_count
        h = _vp()
        check(lib.fpg_convection_create(ctx.h, level_count, ctypes.byref(h)), "fpg_convection_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_convection_destroy(self.h)
        except Exception:
            pass

    def set_matrix(self, matrix, level_interfaces_m, stream=None):
        m = matrix.coefficients_column_major if isinstance(matrix, ConvectiveRedistributionMatrix) else matrix
        m = np.ascontiguousarray(m, np.float32)
        iface = np.ascontiguousarray(level_interfaces_m, np.float32)
        check(lib.fpg_convection_set_matrix(self.h, _p(m), m.size, _p(iface), iface.size, stream),
              "fpg_convection_set_matrix")

    def heights(self) -> np.ndarray:
        out = np.empty(self.level_count, np.float32)
        check(lib.fpg_convection_heights(self.h, _p(out)), "fpg_convection_heights")
        return out

    def apply(self, particles: Particles, stream=None):
        check(lib.fpg_convective_mixing(self.ctx.h, particles.h, self.h, stream), "fpg_convective_mixing")


def dispatch_convective_mixing_gpu(ctx: Context, particles: Particles, level_interfaces_m,
                                   matrix: ConvectiveRedistributionMatrix, stream=None) -> ConvectiveMixing:
    """dispatch_convective_mixing_gpu (src/gpu/convection.rs:68-250) in one
    call; returns the device matrix so later steps can reuse it."""
    L = matrix.level_count()
    iface = np.asarray(level_interfaces_m, np.float32)
    if L == 0:
        raise FpgError(-3, "dispatch_convective_mixing_gpu: invalid level count 0")
    if iface.size != L + 1:
        raise FpgError(-5, f"dispatch_convective_mixing_gpu: expected {L + 1} level interfaces, got {iface.size}")
    cm = ConvectiveMixing(ctx, L)
    cm.set_matrix(matrix, iface, stream)
    cm.apply(particles, stream)
    return cm
