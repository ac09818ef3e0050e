"""FP64 restatement of the source inversion's forward map (TEST
INFRASTRUCTURE ONLY).

The forward of include/fpg_adjoint.h for each source: the forward time loop
of one release alone (release lattice, Philox counters advanced by the
source's particle count x blocks per step, alpha, surface lerp + PBL, the
production step of oracle_core.inc), with a wind bias added to every met
node, followed at every sampling step by the receptors' cloud-in-cell x
vertical-ramp weights.  Unlike oracle/forward.py the release positions and
masses stay in double (no f32 rounding of the initial state), so that
central differences with small steps give the derivative of the FP64 map:
the reference gradient the device adjoint is checked against.  The
reference has no adjoint; this map is the restatement of the device's
forward (csrc/adjoint.cu, csrc/batch.cu) in double.
"""
from __future__ import annotations

import numpy as np

from . import orc


def _cic(x, y, z, nx, ny, ztop, ramp):
    xs, ys = x - 0.5, y - 0.5
    fi, fj = np.floor(xs), np.floor(ys)
    wx1, wy1 = xs - fi, ys - fj
    v = np.clip((ztop + 0.5 * ramp - z) / ramp, 0.0, 1.0)
    return fi.astype(np.int64), fj.astype(np.int64), (1.0 - wx1, wx1), (1.0 - wy1, wy1), v


class OracleInversion:
    def __init__(self, inv, frames, dtype=np.float64, threads=0):
        from flexpart_gpu import synthetic

        self.inv = inv
        self.ens = inv.ensemble
        self.frames = frames
        self.dtype = np.dtype(dtype)
        spec = self.ens.met
        self.spec = spec
        self.heights = synthetic.level_heights(spec.nz, spec.top_m)
        self.xs, self.ys, self.zs = synthetic.velocity_scale(spec)
        self.threads = threads
        self.rmap = -np.ones((max(inv.instance) + 1, spec.nx, spec.ny), np.int64)
        for r, (inst, i, j) in enumerate(inv.receptors):
            self.rmap[inst, i, j] = r

    def _sample(self, sim, state, n, inst):
        spec = self.spec
        x = state.cell_x[:n].astype(np.float64) + state.pos_x[:n].astype(np.float64)
        y = state.cell_y[:n].astype(np.float64) + state.pos_y[:n].astype(np.float64)
        z = state.pos_z[:n].astype(np.float64)
        m = state.mass[0, :n].astype(np.float64)
        act = (state.flags[:n] & 1) != 0
        i0, j0, wx, wy, v = _cic(x, y, z, spec.nx, spec.ny, self.inv.receptor_top_m, self.inv.receptor_ramp_m)
        for di in (0, 1):
            for dj in (0, 1):
                i, j = i0 + di, j0 + dj
                ok = act & (i >= 0) & (j >= 0) & (i < spec.nx) & (j < spec.ny)
                r = np.full(n, -1, np.int64)
                r[ok] = self.rmap[inst, i[ok], j[ok]]
                hit = r >= 0
                np.add.at(sim, r[hit], (m * wx[di] * wy[dj] * v)[hit])

    def forward(self, mass, position, wind_bias=None):
        """sim_r for source masses (kg), release-box lower corners (lon, lat,
        z) and a wind bias of shape (nx, ny, nz, 3) or None."""
        from flexpart_gpu import synthetic
        from flexpart_gpu.records import StepParams

        ens, spec = self.ens, self.spec
        sim = np.zeros(len(self.inv.receptors), np.float64)
        bias = None if wind_bias is None else np.asarray(wind_bias, np.float64).reshape(-1)
        dry = ens.dry_velocity
        for s, src in enumerate(ens.sources):
            n_cap = src.particle_count
            st = orc.State(n_cap, self.dtype)
            lon0, lat0, z0 = (float(v) for v in position[s])
            lon_span = (src.lon if src.lon_max is None else src.lon_max) - src.lon
            lat_span = (src.lat if src.lat_max is None else src.lat_max) - src.lat
            z_span = src.z_max - src.z_min
            m0 = float(mass[s]) / float(n_cap)
            released = 0
            counter = [0, 0, 0, 0]
            t = ens.start
            k = 0
            c = max(int(np.ceil(np.cbrt(np.float64(n_cap)))), 1)
            nxy = max(c * c, 1)
            nzl = max((n_cap + nxy - 1) // nxy, 1)
            while t <= ens.end:
                target = orc.target_emitted_count(n_cap, src.start, src.end, t, released)
                if target > released:
                    idx = np.arange(released, target, dtype=np.int64)
                    fx = ((idx % c) + 0.5) / c
                    fy = (((idx // c) % c) + 0.5) / c
                    fz = (((idx // nxy) % nzl) + 0.5) / nzl
                    x = (lon0 + fx * lon_span - spec.xlon0) / spec.dx_deg
                    y = (lat0 + fy * lat_span - spec.ylat0) / spec.dy_deg
                    fxf, fyf = np.floor(x), np.floor(y)
                    st.cell_x[released:target] = fxf.astype(np.int32)
                    st.cell_y[released:target] = fyf.astype(np.int32)
                    st.pos_x[released:target] = x - fxf
                    st.pos_y[released:target] = y - fyf
                    st.pos_z[released:target] = z0 + fz * z_span
                    st.flags[released:target] = 1
                    st.mass[0, released:target] = m0
                    released = int(target)
                fa, fb, ta, tb = synthetic.bracket_frames(ens, t)
                _, alpha = orc.interpolation_alpha(ta, tb, t, True)
                f0, f1 = self.frames[fa], self.frames[fb]
                pbl = orc.pbl_diagnostics(f0["surface"], f1["surface"], alpha, spec.nx, spec.ny, dtype=self.dtype)
                met = {"u0": f0["u"], "v0": f0["v"], "w0": f0["w"], "u1": f1["u"], "v1": f1["v"], "w1": f1["w"],
                       "heights": self.heights}
                prm = StepParams.production(alpha=alpha, dt_seconds=float(ens.dt), turb_dt_seconds=float(ens.dt),
                                            x_grid_per_meter=self.xs, y_grid_per_meter=self.ys,
                                            z_grid_per_meter=self.zs, key=ens.keys[s], counter=counter,
                                            dry_mode=0 if dry == 0.0 else 1, dry_velocity_m_s=dry, wet_mode=0)
                if released:
                    orc.step(st, released, met, pbl, prm, threads=self.threads, wind_bias=bias)
                counter = orc.next_counter(counter, n_cap, 4)
                if self.inv.sample_every and (k + 1) % self.inv.sample_every == 0 and released:
                    self._sample(sim, st, released, self.inv.instance[s])
                k += 1
                t += ens.dt
        return sim
