"""Shared fixtures: synthetic inputs, and running the same step on the GPU
library and on the oracle."""
from __future__ import annotations

import numpy as np

from flexpart_gpu import synthetic
from flexpart_gpu.records import PARTICLE_DTYPE, StepParams
from oracle import orc

# Tolerance of the floating-point fields after one step: relative 1e-5 (an
# absolute 1e-5 for values below 1).  Integer fields, Philox outputs, alive
# masks, compaction order and grid cell indices are compared bit for bit.
REL_TOL = 1e-5


def close(gpu, ref, rel=REL_TOL):
    gpu = np.asarray(gpu, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(gpu - ref) <= rel * np.maximum(np.abs(ref), 1.0)


def small_met(nx=24, ny=18, nz=12, seed=5, heights=True):
    spec = synthetic.MetSpec(nx=nx, ny=ny, nz=nz, dx_deg=0.5, dy_deg=0.5, xlon0=0.0, ylat0=40.0, n_frames=2,
                             seed=seed)
    frames = synthetic.make_frames(spec)
    hts = synthetic.level_heights(nz, 6000.0) if heights else np.zeros(nz, np.float32)
    met = {"u0": frames[0]["u"], "v0": frames[0]["v"], "w0": frames[0]["w"],
           "u1": frames[1]["u"], "v1": frames[1]["v"], "w1": frames[1]["w"], "heights": hts}
    return spec, frames, met


def population(nx, ny, n, seed=11, inactive_every=7, z_max=2500.0):
    """Particles spread over the domain, a share inactive, with edge cases:
    on the last cell, above the PBL, near the ground, at the top."""
    rng = np.random.default_rng(seed)
    rec = np.zeros(n, PARTICLE_DTYPE)
    x = rng.uniform(0, nx - 1, n)
    y = rng.uniform(0, ny - 1, n)
    fx, fy = np.floor(x), np.floor(y)
    rec["cell_x"] = fx.astype(np.int32)
    rec["cell_y"] = fy.astype(np.int32)
    rec["pos_x"] = (x - fx).astype(np.float32)
    rec["pos_y"] = (y - fy).astype(np.float32)
    rec["pos_z"] = rng.uniform(0.0, z_max, n).astype(np.float32)
    rec["flags"] = 1
    if inactive_every:
        rec["flags"][::inactive_every] = 0
    rec["mass"][:, 0] = rng.uniform(1e-6, 1e-3, n).astype(np.float32)
    rec["turb_u"] = rng.normal(0, 0.6, n).astype(np.float32)
    rec["turb_v"] = rng.normal(0, 0.6, n).astype(np.float32)
    rec["turb_w"] = rng.normal(0, 0.3, n).astype(np.float32)
    if n > 10:
        rec["cell_x"][1], rec["pos_x"][1] = nx - 1, 0.0          # last cell
        rec["cell_y"][2], rec["pos_y"][2] = ny - 1, 0.0
        rec["pos_z"][3] = 0.005                                  # below the reflection floor
        rec["pos_z"][4] = 9000.0                                 # far above the PBL
        rec["pos_z"][5] = 0.0
        rec["cbt"][6] = 1
        rec["mass"][8, 1] = 0.25                                 # a second species
    return rec


def pbl_arrays(frames, alpha, nx, ny, dtype=np.float32):
    return orc.pbl_diagnostics(frames[0]["surface"], frames[1]["surface"], alpha, nx, ny, dtype=dtype)


def oracle_step(rec, met, pbl, params, dtype=np.float32, **kw):
    s = orc.State.from_records(rec, dtype)
    orc.step(s, len(rec), met, pbl, params, **kw)
    return s


def production_params(**kw) -> StepParams:
    base = dict(alpha=0.3, dt_seconds=900.0, turb_dt_seconds=900.0, key=(42, 0), counter=(0, 0, 0, 0),
                dry_mode=1, dry_velocity_m_s=0.002)
    base.update(kw)
    return StepParams.production(**base)
