"""Oracle forward time loop (TEST INFRASTRUCTURE ONLY).

Restates ForwardTimeLoopDriver::run_timestep (src/simulation/timeloop.rs:
915-1316) over the oracle's functions: release (release/mod.rs:90-275,
coords/mod.rs:92-178), interpolation alpha (timeloop.rs:2086-2120), surface
lerp + PBL diagnostics per cell, the four per-particle passes, the Philox
counter advance by dispatch_count * blocks (gpu/langevin_fused.rs:229-233),
optional compaction and spatial reorder.
"""
from __future__ import annotations

import numpy as np

from . import orc


class OracleForward:
    def __init__(self, scn, capacity, frames, dtype=np.float32, sort_interval=0, use_compaction=False,
                 threads=0, key=None, counter=(0, 0, 0, 0), n_substeps=4):
        from flexpart_gpu import synthetic

        self.scn = scn
        self.capacity = capacity
        self.frames = frames
        self.dtype = np.dtype(dtype)
        self.heights = synthetic.level_heights(scn.met.nz, scn.met.top_m)
        self.xs, self.ys, self.zs = synthetic.velocity_scale(scn.met)
        self.rec = np.zeros(capacity, orc.PARTICLE_DTYPE)      # release bookkeeping / cold fields
        self.state = orc.State(capacity, self.dtype)
        self.released = [0] * len(scn.sources)
        self.next_free = 0
        self.active = 0
        self.t = scn.start
        self.step_index = 0
        self.counter = list(counter)
        self.key = tuple(scn.key if key is None else key)
        self.sort_interval = sort_interval
        self.use_compaction = use_compaction
        self.threads = threads
        self.n_substeps = n_substeps

    @property
    def has_remaining_steps(self):
        return self.t <= self.scn.end

    def _release(self, now):
        spec = self.scn.met
        domain = (spec.xlon0, spec.ylat0, spec.dx_deg, spec.dy_deg, spec.nx, spec.ny)
        new = []
        for k, src in enumerate(self.scn.sources):
            target = orc.target_emitted_count(src.particle_count, src.start, src.end, now, self.released[k])
            if target <= self.released[k]:
                continue
            idx = np.arange(self.released[k], target, dtype=np.uint64)
            lon_max = src.lon if src.lon_max is None else src.lon_max
            lat_max = src.lat if src.lat_max is None else src.lat_max
            # ReleaseBounds::sample_stratified (release/mod.rs:256-275), vectorised in f64
            c = float(np.ceil(np.cbrt(np.float64(src.particle_count))))
            nx = max(int(c), 1)
            nxy = max(nx * nx, 1)
            nz = max((src.particle_count + nxy - 1) // nxy, 1)
            ix = idx % np.uint64(nx)
            iy = (idx // np.uint64(nx)) % np.uint64(nx)
            iz = (idx // np.uint64(nxy)) % np.uint64(nz)
            fx = (ix.astype(np.float64) + 0.5) / float(nx)
            fy = (iy.astype(np.float64) + 0.5) / float(nx)
            fz = (iz.astype(np.float64) + 0.5) / float(nz)
            lon = src.lon + fx * (lon_max - src.lon)
            lat = src.lat + fy * (lat_max - src.lat)
            z = src.z_min + fz * (src.z_max - src.z_min)
            x = (lon - domain[0]) / domain[2]
            y = (lat - domain[1]) / domain[3]
            assert np.all((x >= 0) & (x < spec.nx - 1) & (y >= 0) & (y < spec.ny - 1)), "release outside grid"
            r = np.zeros(len(idx), orc.PARTICLE_DTYPE)
            fxf, fyf = np.floor(x), np.floor(y)
            r["cell_x"] = fxf.astype(np.int32)
            r["cell_y"] = fyf.astype(np.int32)
            r["pos_x"] = (x - fxf).astype(np.float32)
            r["pos_y"] = (y - fyf).astype(np.float32)
            r["pos_z"] = z.astype(np.float32)
            r["flags"] = 1
            r["mass"][:, 0] = np.float32(src.mass_kg / float(src.particle_count))
            r["time"] = np.int32(now)
            r["time_mem"] = np.int32(now)
            r["release_point"] = k
            new.append(r)
            self.released[k] = int(target)
        if not new:
            return 0
        r = np.concatenate(new)
        a, b = self.next_free, self.next_free + len(r)
        assert b <= self.capacity, "store full"
        self.rec[a:b] = r
        s = orc.State.from_records(r, self.dtype)
        for f in ("cell_x", "cell_y", "flags", "cbt", "pos_x", "pos_y", "pos_z", "vel_u", "vel_v", "vel_w",
                  "turb_u", "turb_v", "turb_w"):
            getattr(self.state, f)[a:b] = getattr(s, f)
        self.state.mass[:, a:b] = s.mass
        self.next_free = b
        self.active += len(r)
        return len(r)

    def records(self):
        """Current state as fpg_particle records (cold fields from release)."""
        out = self.state.to_records()
        for f in ("time", "time_mem", "release_point", "class_id", "timestep", "time_split"):
            out[f] = self.rec[f]
        return out

    def _apply_perm(self, perm, n):
        rec = self.records()
        rec[:n] = rec[:n][perm]
        self.rec[:n] = self.rec[:n][perm]
        s = orc.State.from_records(rec, self.dtype) if self.dtype == np.float32 else None
        if s is None:
            for f in ("cell_x", "cell_y", "flags", "cbt", "pos_x", "pos_y", "pos_z", "vel_u", "vel_v", "vel_w",
                      "turb_u", "turb_v", "turb_w"):
                getattr(self.state, f)[:n] = getattr(self.state, f)[:n][perm]
            self.state.mass[:, :n] = self.state.mass[:, :n][:, perm]
        else:
            self.state = s

    def run_timestep(self, forcing: dict, wet_cells=None):
        from flexpart_gpu import synthetic
        from flexpart_gpu.records import StepParams

        scn = self.scn
        if self.sort_interval and self.step_index % self.sort_interval == 0 and self.next_free > 0:
            keys = orc.cell_keys(self.state, self.next_free, self.heights, (scn.met.nx, scn.met.ny, scn.met.nz))
            self._apply_perm(np.argsort(keys, kind="stable"), self.next_free)
        released = self._release(self.t)
        fa, fb, ta, tb = synthetic.bracket_frames(scn, self.t)
        st, alpha = orc.interpolation_alpha(ta, tb, self.t, True)
        assert st == 0
        f0, f1 = self.frames[fa], self.frames[fb]
        pbl = orc.pbl_diagnostics(f0["surface"], f1["surface"], alpha, scn.met.nx, scn.met.ny, dtype=self.dtype)
        met = {"u0": f0["u"], "v0": f0["v"], "w0": f0["w"], "u1": f1["u"], "v1": f1["v"], "w1": f1["w"],
               "heights": self.heights}
        dry = forcing.get("dry_velocity", 0.0)
        prm = StepParams.production(alpha=alpha, dt_seconds=float(scn.dt), turb_dt_seconds=float(scn.dt),
                                    x_grid_per_meter=self.xs, y_grid_per_meter=self.ys, z_grid_per_meter=self.zs,
                                    key=self.key, counter=self.counter, n_substeps=self.n_substeps,
                                    rho_grad_over_rho=forcing.get("rho_grad_over_rho", 0.0),
                                    dry_mode=0 if dry == 0.0 else 1, dry_velocity_m_s=dry,
                                    wet_mode=3 if wet_cells is not None else 0)
        kw = {}
        if wet_cells is not None:
            kw = dict(wet_cells_lf=wet_cells, wet_shape=(scn.met.nx, scn.met.ny))
        orc.step(self.state, self.next_free, met, pbl, prm, threads=self.threads, **kw)
        ref_dispatch = self.active if self.use_compaction else self.capacity
        self.counter = orc.next_counter(self.counter, ref_dispatch, self.n_substeps)
        if self.use_compaction:
            rec, count, _ = orc.compact_records(self.records())
            self.rec[:] = rec
            self.state = orc.State.from_records(rec, self.dtype)
            self.active = count
            self.next_free = count
        self.step_index += 1
        t = self.t
        self.t += scn.dt
        return {"time": t, "alpha": alpha, "released": released, "active": self.active, "counter": list(self.counter)}

    def grid(self, species=0, mass_scale=1e6):
        return orc.grid(self.state, self.next_free, species, mass_scale, self.scn.outheights, self.scn.out_shape)


class OracleBackward(OracleForward):
    """BackwardTimeLoopDriver::run_timestep (src/simulation/timeloop.rs:
    1598-1821) over the oracle: receptors are point releases at the start
    time (build_receptor_release_configs, :1896-1917), the clock runs back by
    dt, advection takes -dt while turbulence and deposition take +dt
    (:1724-1746), the counter advances by capacity x blocks, and after the
    step collect_source_collections (:1865-1894) counts the active particles
    inside each region and sums their species-0 mass (in float, slot order,
    as the reference; and in double).  `bracket(t)` gives (frame t0, frame t1,
    time t0, time t1) for the step's time."""

    def __init__(self, scn, capacity, frames, regions, bracket, **kw):
        super().__init__(scn, capacity, frames, **kw)
        self.regions = regions
        self.bracket = bracket

    @property
    def has_remaining_steps(self):
        return self.t >= self.scn.end

    def collections(self):
        spec = self.scn.met
        n = self.next_free
        st = self.state
        act = (st.flags[:n] & 1) != 0
        lon = spec.xlon0 + (st.cell_x[:n].astype(np.float64) + st.pos_x[:n].astype(np.float32).astype(np.float64)) * spec.dx_deg
        lat = spec.ylat0 + (st.cell_y[:n].astype(np.float64) + st.pos_y[:n].astype(np.float32).astype(np.float64)) * spec.dy_deg
        z = st.pos_z[:n].astype(np.float32).astype(np.float64)
        m32 = st.mass[0, :n].astype(np.float32)
        out = []
        for r in self.regions:
            hit = act & (lon >= r["lon_min"]) & (lon <= r["lon_max"]) & (lat >= r["lat_min"]) & \
                (lat <= r["lat_max"]) & (z >= r["z_min_m"]) & (z <= r["z_max_m"])
            s32 = np.float32(0.0)
            for v in m32[hit]:
                s32 = np.float32(s32 + v)
            out.append((int(hit.sum()), float(s32), float(m32[hit].astype(np.float64).sum())))
        return out

    def run_timestep(self, forcing: dict, wet_cells=None):
        from flexpart_gpu.records import StepParams

        scn = self.scn
        released = self._release(self.t)
        f0, f1, ta, tb = self.bracket(self.t)
        st, alpha = orc.interpolation_alpha(ta, tb, self.t, True)
        assert st == 0
        pbl = orc.pbl_diagnostics(f0["surface"], f1["surface"], alpha, scn.met.nx, scn.met.ny, dtype=self.dtype)
        met = {"u0": f0["u"], "v0": f0["v"], "w0": f0["w"], "u1": f1["u"], "v1": f1["v"], "w1": f1["w"],
               "heights": self.heights}
        dry = forcing.get("dry_velocity", 0.0)
        prm = StepParams.production(alpha=alpha, dt_seconds=-float(scn.dt), turb_dt_seconds=float(scn.dt),
                                    x_grid_per_meter=self.xs, y_grid_per_meter=self.ys, z_grid_per_meter=self.zs,
                                    key=self.key, counter=self.counter, n_substeps=self.n_substeps,
                                    rho_grad_over_rho=forcing.get("rho_grad_over_rho", 0.0),
                                    dry_mode=0 if dry == 0.0 else 1, dry_velocity_m_s=dry,
                                    wet_mode=3 if wet_cells is not None else 0)
        kw = {}
        if wet_cells is not None:
            kw = dict(wet_cells_lf=wet_cells, wet_shape=(scn.met.nx, scn.met.ny))
        orc.step(self.state, self.next_free, met, pbl, prm, threads=self.threads, **kw)
        self.counter = orc.next_counter(self.counter, self.capacity, self.n_substeps)
        self.step_index += 1
        t = self.t
        self.t -= scn.dt
        return {"time": t, "alpha": alpha, "released": released, "active": self.active,
                "counter": list(self.counter), "collections": self.collections()}
