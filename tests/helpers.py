"""Shared fixtures: synthetic inputs, and running the same step on the GPU
library and on the oracle."""
from __future__ import annotations

import numpy as np

from flexpart_gpu import synthetic
from flexpart_gpu.records import PARTICLE_DTYPE, StepParams
from oracle import orc

# Tolerance of the floating-point fields after one step: relative 1e-5 of the
# field's scale.  The scale is the value itself, floored where a field's value
# is the small difference of large terms:
#   grid coordinates: max(|x|, 1 cell);
#   heights: max(|z|, |z at step start|, 100 m) -- a particle reflected at
#     the PBL top computes 2h - z with h ~ 1e3 m, so its height carries an
#     absolute rounding of ulp(h) ~ 1e-4 m however small z ends up (the FP32
#     oracle differs from the FP64 one by up to 7e-5 relative at z = 4.5 m);
#   turbulent and mean velocities: max(|v|, 2 m/s) -- each sub-step adds
#     an Ornstein-Uhlenbeck decay, a noise term of size sigma_w (up to ~2 m/s
#     for w* <= 2.5 m/s) and a drift term whose height derivative is steep
#     near the ground, so a velocity near zero is the difference of terms of
#     that size (the FP32 oracle differs from the FP64 one by up to 2e-5 m/s);
#   masses: the value itself.
# Integer fields, Philox outputs, alive masks, compaction order and grid cell
# indices are compared bit for bit.
REL_TOL = 1e-5


def close(gpu, ref, rel=REL_TOL, floor=1.0):
    gpu = np.asarray(gpu, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(gpu - ref) <= rel * np.maximum(np.abs(ref), floor)


def _fields(rec_or_state):
    """float64 views of the compared fields of records or an oracle State."""
    if isinstance(rec_or_state, np.ndarray):
        r = rec_or_state
        out = {"grid_x": r["cell_x"].astype(np.float64) + r["pos_x"],
               "grid_y": r["cell_y"].astype(np.float64) + r["pos_y"]}
        for f in ("pos_z", "turb_u", "turb_v", "turb_w", "vel_u", "vel_v", "vel_w"):
            out[f] = r[f].astype(np.float64)
        for k in range(4):
            out[f"mass{k}"] = r["mass"][:, k].astype(np.float64)
        return out
    s = rec_or_state
    out = {"grid_x": s.cell_x.astype(np.float64) + s.pos_x, "grid_y": s.cell_y.astype(np.float64) + s.pos_y}
    for f in ("pos_z", "turb_u", "turb_v", "turb_w", "vel_u", "vel_v", "vel_w"):
        out[f] = np.asarray(getattr(s, f), np.float64)
    for k in range(4):
        out[f"mass{k}"] = np.asarray(s.mass[k], np.float64)
    return out


ENVELOPE = 4.0
# Largest share of the active particles a floating-point field may pass
# through the FP64 envelope alone (below one particle in 10 000; none in a
# population of fewer than 10 000 active particles).
MAX_ENVELOPE_SHARE = 1e-4


def field_checks(g, s, z_in, s64=None, stats=None):
    """Per-field parity masks of GPU records `g` against the FP32 oracle
    state `s`.  With the FP64 oracle state `s64`, a particle also passes when
    the GPU is no further from the FP32 oracle than ENVELOPE times the FP32
    oracle's own distance from FP64: for the few ill-conditioned particles
    (unstable cells, a start near the ground) FP32 arithmetic itself cannot
    resolve the step to 1e-5, and the GPU is then held to FP32's own
    accuracy.  `stats` (a dict) counts those particles per field."""
    G, S = _fields(g), _fields(s)
    S64 = _fields(s64) if s64 is not None else None
    zscale = np.maximum(np.maximum(np.abs(S["pos_z"]), np.abs(z_in.astype(np.float64))), 100.0)
    floors = {"grid_x": 1.0, "grid_y": 1.0}
    out = {}
    for f in G:
        if f == "pos_z":
            ok = np.abs(G[f] - S[f]) <= REL_TOL * zscale
        elif f.startswith("mass"):
            ok = close(G[f], S[f], floor=0.0)
        elif f.startswith("turb") or f.startswith("vel"):
            ok = close(G[f], S[f], floor=2.0)
        else:
            ok = close(G[f], S[f], floor=floors[f])
        if S64 is not None:
            env = np.abs(G[f] - S[f]) <= ENVELOPE * np.abs(S[f] - S64[f]) + 1e-12
            if stats is not None:
                stats[f] = stats.get(f, 0) + int((~ok & env).sum())
            ok = ok | env
        out[f] = ok
    return out


def assert_parity(g, s, z_in, s64, label, n_active=None, max_share=MAX_ENVELOPE_SHARE):
    """Every floating-point field within tolerance (field_checks), at most
    `max_share` of the active particles passing through the FP64 envelope
    per field, and the integer fields (flags, cbt) bit-exact.  Returns the
    envelope counts per field."""
    stats = {}
    checks = field_checks(g, s, z_in, s64, stats)
    for k, ok in checks.items():
        if not ok.all():
            bad = np.flatnonzero(~ok)[:5]
            detail = [(int(i), float(z_in[i]), float(g["pos_z"][i]), float(np.asarray(s.pos_z)[i]),
                       float(g["turb_w"][i]), float(np.asarray(s.turb_w)[i])) for i in bad]
            raise AssertionError(f"{label}: {k} differs at (slot, z_in, z_gpu, z_orc, tw_gpu, tw_orc) {detail}")
    if n_active is None:
        n_active = int((np.asarray(s.flags) & 1).sum())
    allowed = int(np.floor(max_share * n_active))
    over = {k: v for k, v in stats.items() if v > allowed}
    assert not over, f"{label}: envelope share above {max_share} of {n_active} active particles: {over}"
    assert np.array_equal(g["flags"], np.asarray(s.flags)), f"{label}: flags"
    assert np.array_equal(g["cbt"], np.asarray(s.cbt)), f"{label}: cbt"
    return stats


FP64_FIELDS = ("grid_x", "grid_y", "pos_z", "turb_u", "turb_v", "turb_w", "mass0")


def fp64_errors(g, s, s64, z_in, active):
    """Max scaled error against the FP64 oracle of the GPU and of the FP32
    oracle, per field, over the active particles (scales as field_checks:
    1 cell, the height scale, 2 m/s, the mass itself)."""
    G, S, D = _fields(g), _fields(s), _fields(s64)
    zs = np.maximum(np.maximum(np.abs(D["pos_z"][active]), np.abs(z_in[active].astype(np.float64))), 100.0)
    floors = {"grid_x": 1.0, "grid_y": 1.0, "turb_u": 2.0, "turb_v": 2.0, "turb_w": 2.0, "mass0": 1e-30}
    out = {}
    for f in FP64_FIELDS:
        ref = D[f][active]
        sc = zs if f == "pos_z" else np.maximum(np.abs(ref), floors[f])
        out[f] = (float(np.max(np.abs(G[f][active] - ref) / sc)), float(np.max(np.abs(S[f][active] - ref) / sc)))
    return out


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
    """Production step settings; the metres->grid scale is that of the
    0.5-degree test grid at 44 N (about 1/40 km and 1/55 km)."""
    base = dict(alpha=0.3, dt_seconds=900.0, turb_dt_seconds=900.0, key=(42, 0), counter=(0, 0, 0, 0),
                dry_mode=1, dry_velocity_m_s=0.002, x_grid_per_meter=2.5e-5, y_grid_per_meter=1.8e-5)
    base.update(kw)
    return StepParams.production(**base)
