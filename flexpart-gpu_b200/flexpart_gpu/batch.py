"""Batch: many release scenarios stepped as one population behind the C ABI
(``fpg_batch_*`` in include/fpg_driver.h).

Each scenario computes what one ForwardTimeLoopDriver with one release,
capacity = its particle count and its own Philox key would compute
(src/simulation/timeloop.rs:915-1316); all scenarios share one met frame ring
and one clock, and one step is one replay of a captured CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import synthetic
from ._lib import check, lib
from .api import Context, Particles
from .records import BatchConfig, BatchScenario, BatchTuning, GridDomain, PblOptions, Release

_vp = ctypes.c_void_p


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class _ParticlesView(Particles):
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = _vp(handle)

    def __del__(self):
        pass


def ensemble_config(ens: synthetic.Ensemble, output_every_steps: int = 0, n_substeps: int = 4,
                    min_height_m: float = 0.01, rho_grad_over_rho: float = 0.0) -> BatchConfig:
    xs, ys, zs = synthetic.velocity_scale(ens.met)
    c = BatchConfig()
    c.start_seconds, c.end_seconds, c.timestep_seconds = ens.start, ens.end, ens.dt
    c.frame_seconds, c.n_frames = ens.met.frame_seconds, ens.met.n_frames
    c.x_grid_per_meter, c.y_grid_per_meter, c.z_grid_per_meter = xs, ys, zs
    c.pbl_options = PblOptions.default()
    c.dry_reference_height_m = 15.0
    c.dry_velocity_m_s = ens.dry_velocity
    c.rho_grad_over_rho = rho_grad_over_rho
    c.n_substeps = n_substeps
    c.min_height_m = min_height_m
    c.wet_from_precipitation = 1 if ens.met.wet else 0
    c.wet_gas_a, c.wet_gas_b = ens.wet_a, ens.wet_b
    m = ens.met
    c.release_grid = GridDomain(m.xlon0, m.ylat0, m.dx_deg, m.dy_deg, m.nx, m.ny)
    c.out_nx, c.out_ny, c.out_nz = ens.out_shape
    c.output_every_steps = output_every_steps
    return c


def ensemble_scenarios(ens: synthetic.Ensemble):
    out = []
    for s, (src, key) in enumerate(zip(ens.sources, ens.keys)):
        r = Release(src.start, src.end, src.lon, src.lon if src.lon_max is None else src.lon_max, src.lat,
                    src.lat if src.lat_max is None else src.lat_max, src.z_min, src.z_max, src.mass_kg,
                    src.particle_count)
        bs = BatchScenario()
        bs.release = r
        bs.key[0], bs.key[1] = key[0] & 0xFFFFFFFF, key[1] & 0xFFFFFFFF
        out.append(bs)
    return out


class Batch:
    def __init__(self, ctx: Context, config: BatchConfig, scenarios, met_shape, level_heights=None,
                 outheights=None):
        self.ctx = ctx
        self.n_scenarios = len(scenarios)
        self.out_shape = (config.out_nx, config.out_ny, config.out_nz)
        self._oh = None if outheights is None else np.ascontiguousarray(outheights, np.float32)
        config.outheights = None if self._oh is None else self._oh.ctypes.data
        arr = (BatchScenario * max(self.n_scenarios, 1))(*scenarios)
        self._heights = None if level_heights is None else np.ascontiguousarray(level_heights, np.float32)
        nx, ny, nz = met_shape
        h = _vp()
        check(lib.fpg_batch_create(ctx.h, ctypes.byref(config), arr, self.n_scenarios, nx, ny, nz,
                                   _p(self._heights), ctypes.byref(h)), "fpg_batch_create")
        self.h = h
        self.config = config

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_batch_destroy(self.h)
        except Exception:
            pass

    def upload_frame(self, k: int, frame: dict, precipitation=None):
        u = np.ascontiguousarray(frame["u"].reshape(-1), np.float32)
        v = np.ascontiguousarray(frame["v"].reshape(-1), np.float32)
        w = np.ascontiguousarray(frame["w"].reshape(-1), np.float32)
        surf = np.ascontiguousarray(frame["surface"])
        pr = None if precipitation is None else np.ascontiguousarray(precipitation, np.float32)
        check(lib.fpg_batch_upload_frame(self.h, k, _p(u), _p(v), _p(w), _p(surf), _p(pr)), "fpg_batch_upload_frame")

    def run(self, n_steps: int, graph: bool = True):
        check(lib.fpg_batch_run(self.h, n_steps, 1 if graph else 0), "fpg_batch_run")

    def run_sequential(self, n_steps: int):
        check(lib.fpg_batch_run_sequential(self.h, n_steps), "fpg_batch_run_sequential")

    @property
    def steps_done(self) -> int:
        return int(lib.fpg_batch_steps_done(self.h))

    def slots(self, s: int):
        first, count = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib.fpg_batch_scenario_slots(self.h, s, ctypes.byref(first), ctypes.byref(count)),
              "fpg_batch_scenario_slots")
        return first.value, count.value

    @property
    def particles(self) -> Particles:
        return _ParticlesView(self.ctx, lib.fpg_batch_particles(self.h))

    def download_grids(self, out=None):
        """The per-scenario grids of the last output step as (counts, scaled
        mass), u32 of shape (n_scenarios, nx, ny, nz); `out` may pass two
        such C-contiguous arrays (page-locked ones copy fastest) to fill."""
        nx, ny, nz = self.out_shape
        shape = (self.n_scenarios, nx, ny, nz)
        if out is None:
            counts, mass = np.zeros(shape, np.uint32), np.zeros(shape, np.uint32)
        else:
            counts, mass = out
            for a in (counts, mass):
                if a.shape != shape or a.dtype != np.uint32 or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"grid output arrays must be C-contiguous uint32 of shape {shape}")
        check(lib.fpg_batch_download_grids(self.h, _p(counts), _p(mass)), "fpg_batch_download_grids")
        return counts, mass

    def autotune(self, reps: int = 3):
        """Times every compiled launch shape on the next step (from a
        snapshot, restored afterwards) and keeps the fastest; returns
        (best, all candidates) as dicts."""
        n = lib.fpg_batch_tuning_candidates(None, 0)
        res = (BatchTuning * n)()
        best = BatchTuning()
        check(lib.fpg_batch_autotune(self.h, reps, res, n, ctypes.byref(best)), "fpg_batch_autotune")
        return best.as_dict(), [r.as_dict() for r in res]

    @property
    def tuning(self) -> dict:
        t = BatchTuning()
        check(lib.fpg_batch_get_tuning(self.h, ctypes.byref(t)), "fpg_batch_get_tuning")
        return t.as_dict()

    @tuning.setter
    def tuning(self, t: dict):
        bt = BatchTuning(t["block_threads"], t["min_blocks_per_sm"], t["particles_per_thread"], t.get("step_ms", 0.0))
        check(lib.fpg_batch_set_tuning(self.h, ctypes.byref(bt)), "fpg_batch_set_tuning")

    def errors(self) -> int:
        f = ctypes.c_int32()
        check(lib.fpg_batch_errors(self.h, ctypes.byref(f)), "fpg_batch_errors")
        return f.value


def tuning_candidates():
    n = lib.fpg_batch_tuning_candidates(None, 0)
    arr = (BatchTuning * n)()
    lib.fpg_batch_tuning_candidates(arr, n)
    return [a.as_dict() for a in arr]


def upload_ensemble_met(batch: Batch, ens: synthetic.Ensemble):
    """Makes and uploads every frame of the ensemble's met ring; returns the
    frames and per-frame precipitation (host arrays)."""
    frames = synthetic.make_frames(ens.met)
    precs = [synthetic.precipitation(ens.met, k) if ens.met.wet else None for k in range(ens.met.n_frames)]
    for k, f in enumerate(frames):
        batch.upload_frame(k, f, precs[k])
    return frames, precs


__all__ = ["Batch", "tuning_candidates", "ensemble_config", "ensemble_scenarios", "upload_ensemble_met", "particle_steps", "target_emitted"]


def target_emitted(src, now: int, released: int) -> int:
    """ReleaseState::target_emitted_count (src/release/mod.rs:181-196)."""
    if now < src.start or now > src.end:
        return released
    if src.start == src.end or now == src.end:
        return src.particle_count
    return src.particle_count * (now - src.start) // (src.end - src.start)


def particle_steps(ens: synthetic.Ensemble, first_step: int = 0, n_steps: int | None = None) -> int:
    """Particle-steps of steps [first_step, first_step + n_steps) of the
    ensemble: each step moves every particle released up to and including
    that step."""
    n_steps = ens.n_steps - first_step if n_steps is None else n_steps
    total = 0
    for src in ens.sources:
        rel = 0
        for k in range(first_step + n_steps):
            rel = max(rel, target_emitted(src, ens.start + k * ens.dt, rel))
            if k >= first_step:
                total += rel
    return total
