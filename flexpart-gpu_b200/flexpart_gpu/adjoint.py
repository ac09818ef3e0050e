"""SourceInversion: the forward/backward pair of include/fpg_adjoint.h.

``forward(mass, position, wind_bias)`` runs the production step for every
source and returns the receptors' time-integrated smooth concentrations;
``backward(d_sim)`` returns dL/dmass, dL/dposition and dL/dwind_bias for
dL/dsim = d_sim, as a differentiable operator's backward does.  There is no
reference counterpart (the reference has no adjoint).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import synthetic
from ._lib import check, lib
from .api import Context
from .batch import ensemble_config, ensemble_scenarios
from .records import InverseConfig, Receptor

_vp = ctypes.c_void_p


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def inversion_config(inv: synthetic.Inversion) -> InverseConfig:
    c = InverseConfig()
    c.batch = ensemble_config(inv.ensemble)
    c.sample_every_steps = inv.sample_every
    c.receptor_top_m = inv.receptor_top_m
    c.receptor_ramp_m = inv.receptor_ramp_m
    c.checkpoint_every = inv.checkpoint_every
    c.tape_tail_windows = inv.tape_tail_windows
    return c


class SourceInversion:
    def __init__(self, ctx: Context, inv: synthetic.Inversion, frames=None, precipitation=None):
        self.ctx = ctx
        self.inv = inv
        ens = inv.ensemble
        spec = ens.met
        self.shape = (spec.nx, spec.ny, spec.nz)
        self.n_sources = len(ens.sources)
        self.n_receptors = len(inv.receptors)
        cfg = inversion_config(inv)
        scen = ensemble_scenarios(ens)
        arr = (type(scen[0]) * self.n_sources)(*scen)
        inst = np.ascontiguousarray(inv.instance, np.uint32)
        rec = (Receptor * max(self.n_receptors, 1))(*[Receptor(*r) for r in inv.receptors])
        heights = synthetic.level_heights(spec.nz, spec.top_m)
        h = _vp()
        check(lib.fpg_inverse_create(ctx.h, ctypes.byref(cfg), arr, _p(inst), self.n_sources, spec.nx, spec.ny,
                                     spec.nz, _p(heights), rec, self.n_receptors, ctypes.byref(h)),
              "fpg_inverse_create")
        self.h = h
        if frames is None:
            frames = synthetic.make_frames_uniform_pbl(spec) if getattr(inv, "smooth", False) \
                else synthetic.make_frames(spec)
        if precipitation is None and spec.wet:
            precipitation = [synthetic.precipitation(spec, k) for k in range(spec.n_frames)]
        self.frames = frames
        for k, f in enumerate(frames):
            pr = None if precipitation is None else np.ascontiguousarray(precipitation[k], np.float32)
            u = np.ascontiguousarray(f["u"].reshape(-1), np.float32)
            v = np.ascontiguousarray(f["v"].reshape(-1), np.float32)
            w = np.ascontiguousarray(f["w"].reshape(-1), np.float32)
            check(lib.fpg_inverse_upload_frame(self.h, k, _p(u), _p(v), _p(w), _p(np.ascontiguousarray(f["surface"])),
                                               _p(pr)), "fpg_inverse_upload_frame")
        self.mass0 = np.array([s.mass_kg for s in ens.sources], np.float64)
        self.position0 = np.array([[s.lon, s.lat, s.z_min] for s in ens.sources], np.float64)

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_inverse_destroy(self.h)
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(lib.fpg_inverse_device_bytes(self.h))

    def forward(self, mass=None, position=None, wind_bias=None) -> np.ndarray:
        m = None if mass is None else np.ascontiguousarray(mass, np.float64)
        p = None if position is None else np.ascontiguousarray(position, np.float64).reshape(-1)
        check(lib.fpg_inverse_set_sources(self.h, _p(m), _p(p)), "fpg_inverse_set_sources")
        b = None if wind_bias is None else np.ascontiguousarray(wind_bias, np.float32).reshape(-1)
        check(lib.fpg_inverse_set_wind_bias(self.h, _p(b)), "fpg_inverse_set_wind_bias")
        sim = np.zeros(max(self.n_receptors, 1), np.float64)
        check(lib.fpg_inverse_forward(self.h, _p(sim)), "fpg_inverse_forward")
        return sim[: self.n_receptors]

    def backward(self, d_sim, want_bias: bool = True, group=None):
        """Gradients of the loss given dL/dsim.  With `group` (a
        torch.distributed group whose ranks each hold a shard of the
        instances), the wind-bias gradient is summed over the ranks in fixed
        point (distributed.allreduce_gradient_fixed_point); the source
        gradients stay per rank."""
        g = np.ascontiguousarray(d_sim, np.float64)
        dm = np.zeros(self.n_sources, np.float64)
        dp = np.zeros((self.n_sources, 3), np.float64)
        nx, ny, nz = self.shape
        db = np.zeros((nx, ny, nz, 3), np.float32) if want_bias else None
        check(lib.fpg_inverse_backward(self.h, _p(g), _p(dm), _p(dp), _p(db)), "fpg_inverse_backward")
        if db is not None and group is not None:
            from .distributed import allreduce_gradient_fixed_point
            db = allreduce_gradient_fixed_point(db, group).astype(np.float32)
        return {"mass": dm, "position": dp, "wind_bias": db}


def misfit(sim, obs):
    """L = sum (sim - obs)^2 and dL/dsim."""
    r = np.asarray(sim) - np.asarray(obs)
    return float(np.sum(r * r)), 2.0 * r


def synthetic_observations(model: SourceInversion, seed: int = 7):
    """Observed values: the forward under the true emissions perturbed by
    lognormal(0, 0.5) factors, plus 10 % Gaussian noise."""
    rng = np.random.default_rng(seed)
    true_mass = model.mass0 * rng.lognormal(0.0, 0.5, model.n_sources)
    sim = model.forward(true_mass, model.position0)
    return sim * (1.0 + 0.1 * rng.standard_normal(sim.size)), true_mass


__all__ = ["SourceInversion", "inversion_config", "misfit", "synthetic_observations"]
