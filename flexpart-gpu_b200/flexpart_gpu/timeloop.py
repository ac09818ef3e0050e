"""ForwardDriver: the forward time loop behind the C ABI (include/fpg_driver.h),
in the shape of the reference's ForwardTimeLoopDriver
(src/simulation/timeloop.rs:660-1431): ``run_timestep(met, forcing)``,
``run_to_end``, ``has_remaining_steps``, ``finalize``,
``accumulate_concentration_grid``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import synthetic
from ._lib import check, lib
from .api import Context, Grid, Particles
from .records import (
    BackwardConfig,
    FORCING_NONE,
    FORCING_PER_CELL,
    FORCING_UNIFORM,
    ForwardConfig,
    Forcing,
    GridDomain,
    MetBracket,
    PblOptions,
    ReceptorRelease,
    Release,
    SourceCollection,
    SourceRegion,
    StepReport,
    StepTiming,
)

_vp = ctypes.c_void_p


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class _ParticlesView(Particles):
    """A Particles object over the driver's own handle (not owned)."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = _vp(handle)

    def __del__(self):
        pass


class ForwardDriver:
    def __init__(self, ctx: Context, config: ForwardConfig, releases, grid: GridDomain, capacity: int,
                 met_shape, level_heights=None):
        self.ctx = ctx
        self.config = config
        rel = (Release * max(len(releases), 1))(*releases)
        nx, ny, nz = met_shape
        self._heights = None if level_heights is None else np.ascontiguousarray(level_heights, np.float32)
        h = _vp()
        check(lib.fpg_forward_create(ctx.h, ctypes.byref(config), rel, len(releases), ctypes.byref(grid), capacity,
                                     nx, ny, nz, _p(self._heights), ctypes.byref(h)), "fpg_forward_create")
        self.h = h
        self.capacity = capacity
        self.met_shape = met_shape
        self._keep = []

    def __del__(self):
        # the driver synchronises its context's stream when destroyed, so it
        # must go before the context (include/fpg_driver.h)
        try:
            if self.h and self.ctx.h:
                lib.fpg_forward_destroy(self.h)
        except Exception:
            pass

    @property
    def has_remaining_steps(self) -> bool:
        return bool(lib.fpg_forward_has_remaining_steps(self.h))

    @property
    def current_time_seconds(self) -> int:
        return int(lib.fpg_forward_current_time(self.h))

    @property
    def particles(self) -> Particles:
        return _ParticlesView(self.ctx, lib.fpg_forward_particles(self.h))

    def run_timestep(self, met: MetBracket, forcing: Forcing) -> StepReport:
        rep = StepReport()
        check(lib.fpg_forward_run_timestep(self.h, ctypes.byref(met), ctypes.byref(forcing), ctypes.byref(rep)),
              "fpg_forward_run_timestep")
        return rep

    def finalize(self):
        check(lib.fpg_forward_finalize(self.h), "fpg_forward_finalize")

    def run_to_end(self, met: MetBracket, forcing: Forcing) -> list[StepReport]:
        """run_to_end (timeloop.rs:1318-1333): every remaining step with one met
        bracket and forcing, then finalize; the steps' reports."""
        reports = []
        while self.has_remaining_steps:
            reports.append(self.run_timestep(met, forcing))
        self.finalize()
        return reports

    def enable_met_ring(self, n_slots: int = 3):
        """Met streaming: a device ring of n_slots frames filled ahead of use."""
        check(lib.fpg_forward_met_ring(self.h, n_slots), "fpg_forward_met_ring")

    def prefetch_frame(self, time_seconds: int, u, v, w, surface):
        """Queues the copy of the met frame valid at time_seconds; the host
        arrays must stay unchanged until the frame is used."""
        self._keep.append((u, v, w, surface))
        if len(self._keep) > 16:
            del self._keep[:-16]
        ptr = lambda a: ctypes.c_void_p(a.ctypes.data) if hasattr(a, "ctypes") else ctypes.c_void_p(int(a))
        check(lib.fpg_forward_prefetch_frame(self.h, time_seconds, ptr(u), ptr(v), ptr(w), ptr(surface)),
              "fpg_forward_prefetch_frame")

    def met_ring_stats(self):
        hits, uploads = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib.fpg_forward_met_ring_stats(self.h, ctypes.byref(hits), ctypes.byref(uploads)),
              "fpg_forward_met_ring_stats")
        return int(hits.value), int(uploads.value)

    def set_profiling(self, on: bool = True):
        """Per-section device timing of every step (each step then waits for
        its device work); also on when FLEXPART_GPU_PROFILE=1 at creation."""
        check(lib.fpg_forward_set_profiling(self.h, 1 if on else 0), "fpg_forward_set_profiling")

    def set_validation_mode(self, on: bool = True):
        """The reference's validation path: separated advection, Hanna-record,
        Langevin and deposition passes (the fused kernel's bits); also on when
        FLEXPART_GPU_VALIDATION=1 at creation."""
        check(lib.fpg_forward_set_validation_mode(self.h, 1 if on else 0), "fpg_forward_set_validation_mode")

    def last_timing(self) -> StepTiming:
        """The timing of the last step run with profiling on."""
        t = StepTiming()
        check(lib.fpg_forward_last_timing(self.h, ctypes.byref(t)), "fpg_forward_last_timing")
        return t

    def accumulate_concentration_grid(self, grid: Grid, species=0, mass_scale=1.0e6, outheights=None):
        oh = None if outheights is None else np.ascontiguousarray(outheights, np.float32)
        check(lib.fpg_forward_accumulate_grid(self.h, grid.h, species, mass_scale, _p(oh),
                                              0 if oh is None else oh.size), "fpg_forward_accumulate_grid")
        return grid.download()


class BackwardDriver:
    """Backward (receptor) mode behind the C ABI, in the shape of the
    reference's BackwardTimeLoopDriver (src/simulation/timeloop.rs:1433-1909):
    ``run_timestep(met, forcing)`` returns the step report and, per source
    region, (hit_count, total_mass_kg, total_mass_kg_f64)."""

    def __init__(self, ctx: Context, config: BackwardConfig, receptors, regions, grid: GridDomain, capacity: int,
                 met_shape, level_heights=None):
        self.ctx = ctx
        self.config = config
        rec = (ReceptorRelease * max(len(receptors), 1))(*receptors)
        reg = (SourceRegion * max(len(regions), 1))(*regions)
        self.n_regions = len(regions)
        nx, ny, nz = met_shape
        self._heights = None if level_heights is None else np.ascontiguousarray(level_heights, np.float32)
        h = _vp()
        check(lib.fpg_backward_create(ctx.h, ctypes.byref(config), rec, len(receptors), reg, len(regions),
                                      ctypes.byref(grid), capacity, nx, ny, nz, _p(self._heights), ctypes.byref(h)),
              "fpg_backward_create")
        self.h = h
        self.capacity = capacity

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_backward_destroy(self.h)
        except Exception:
            pass

    @property
    def has_remaining_steps(self) -> bool:
        return bool(lib.fpg_backward_has_remaining_steps(self.h))

    @property
    def current_time_seconds(self) -> int:
        return int(lib.fpg_backward_current_time(self.h))

    @property
    def particles(self) -> Particles:
        return _ParticlesView(self.ctx, lib.fpg_backward_particles(self.h))

    def run_timestep(self, met: MetBracket, forcing: Forcing):
        rep = StepReport()
        col = (SourceCollection * max(self.n_regions, 1))()
        check(lib.fpg_backward_run_timestep(self.h, ctypes.byref(met), ctypes.byref(forcing), ctypes.byref(rep),
                                            col), "fpg_backward_run_timestep")
        return rep, [(int(c.hit_count), float(c.total_mass_kg), float(c.total_mass_kg_f64))
                     for c in col[: self.n_regions]]

    def set_validation_mode(self, on: bool = True):
        """The separated passes the reference's backward driver always runs
        (timeloop.rs:1433-1437); the fused kernel's bits."""
        check(lib.fpg_backward_set_validation_mode(self.h, 1 if on else 0), "fpg_backward_set_validation_mode")

    def run_to_end(self, met: MetBracket, forcing: Forcing):
        """run_to_end (timeloop.rs:1828-1838): every remaining step with one met
        bracket and forcing; the steps' (report, collections) pairs."""
        out = []
        while self.has_remaining_steps:
            out.append(self.run_timestep(met, forcing))
        return out


def backward_config(**kw) -> BackwardConfig:
    c = BackwardConfig()
    lib.fpg_backward_config_default(ctypes.byref(c))
    for k, v in kw.items():
        if k in ("philox_key", "initial_philox_counter"):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = int(x) & 0xFFFFFFFF
        else:
            setattr(c, k, v)
    return c


def default_config(**kw) -> ForwardConfig:
    c = ForwardConfig()
    lib.fpg_forward_config_default(ctypes.byref(c))
    for k, v in kw.items():
        if k in ("philox_key", "initial_philox_counter"):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = int(x) & 0xFFFFFFFF
        else:
            setattr(c, k, v)
    return c


def parse_timestamp(s: str) -> int:
    out = ctypes.c_int64()
    check(lib.fpg_parse_timestamp(s.encode(), ctypes.byref(out)), "fpg_parse_timestamp")
    return out.value


# ---- scenario plumbing -----------------------------------------------------

def scenario_releases(scn: synthetic.Scenario):
    out = []
    for s in scn.sources:
        out.append(Release(s.start, s.end, s.lon, s.lon if s.lon_max is None else s.lon_max, s.lat,
                           s.lat if s.lat_max is None else s.lat_max, s.z_min, s.z_max, s.mass_kg, s.particle_count))
    return out


def scenario_domain(scn: synthetic.Scenario) -> GridDomain:
    m = scn.met
    return GridDomain(m.xlon0, m.ylat0, m.dx_deg, m.dy_deg, m.nx, m.ny)


def scenario_config(scn: synthetic.Scenario, **kw) -> ForwardConfig:
    xs, ys, zs = synthetic.velocity_scale(scn.met)
    base = dict(start_seconds=scn.start, end_seconds=scn.end, timestep_seconds=scn.dt, x_grid_per_meter=xs,
                y_grid_per_meter=ys, z_grid_per_meter=zs, philox_key=scn.key)
    base.update(kw)
    return default_config(**base)


class BracketSource:
    """Builds the MetBracket of a scenario at time t from its frame ring
    (host arrays kept alive here)."""

    def __init__(self, scn: synthetic.Scenario, frames):
        self.scn = scn
        self.frames = [{k: np.ascontiguousarray(f[k].reshape(-1)) for k in ("u", "v", "w")} | {"surface": f["surface"]}
                       for f in frames]

    def at(self, t: int) -> MetBracket:
        fa, fb, ta, tb = synthetic.bracket_frames(self.scn, t)
        a, b = self.frames[fa], self.frames[fb]
        return MetBracket(a["u"].ctypes.data, a["v"].ctypes.data, a["w"].ctypes.data, b["u"].ctypes.data,
                          b["v"].ctypes.data, b["w"].ctypes.data, a["surface"].ctypes.data,
                          b["surface"].ctypes.data, ta, tb)


def uniform_forcing(dry_velocity=0.0, wet_lambda=0.0, wet_fraction=0.0, rho_grad_over_rho=0.0) -> Forcing:
    f = Forcing()
    f.dry_mode = FORCING_UNIFORM
    f.dry_velocity_m_s = dry_velocity
    f.wet_mode = FORCING_UNIFORM
    f.wet_lambda_s_inv = wet_lambda
    f.wet_fraction = wet_fraction
    f.rho_grad_over_rho = rho_grad_over_rho
    return f


def cell_forcing(cells, dry_velocity=0.0, rho_grad_over_rho=0.0) -> Forcing:
    f = uniform_forcing(dry_velocity, 0.0, 0.0, rho_grad_over_rho)
    f.wet_mode = FORCING_PER_CELL
    f.wet_cells = cells.h.value
    return f


__all__ = ["ForwardDriver", "BackwardDriver", "backward_config", "default_config", "parse_timestamp", "scenario_releases", "scenario_domain",
           "scenario_config", "BracketSource", "uniform_forcing", "cell_forcing", "FORCING_NONE", "PblOptions"]
