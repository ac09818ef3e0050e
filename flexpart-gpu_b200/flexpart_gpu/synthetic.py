"""Seeded synthetic inputs of the benchmark configurations.

No public dataset is involved: the meteorology, sources and surface fields
are drawn from the value distributions the configurations state
(u, v ~ N(5, 3) m/s smoothed by a Gaussian filter of sigma 3 cells and
renormalised to those moments, w ~ N(0, 0.05) m/s, PBL height U(300, 1500) m,
u* U(0.1, 0.6) m/s, 1/L ~ N(0, 0.01) 1/m, temperature from a 6.5 K/km lapse
rate, precipitation lognormal(-1, 1) mm/h on 30 % of cells), with a fixed
numpy seed per configuration, so every run and every process sees the same
arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .records import PARTICLE_DTYPE, SURFACE_DTYPE

R_EARTH = 6_371_000.0  # src/bin/fortran-validation.rs:21


@dataclass
class MetSpec:
    nx: int
    ny: int
    nz: int
    dx_deg: float
    dy_deg: float
    xlon0: float
    ylat0: float
    top_m: float = 15_000.0
    n_frames: int = 2
    frame_seconds: int = 3 * 3600
    seed: int = 0
    wet: bool = False


@dataclass
class Source:
    lon: float
    lat: float
    z_min: float
    z_max: float
    mass_kg: float
    particle_count: int
    start: int  # seconds since epoch
    end: int
    lon_max: float | None = None
    lat_max: float | None = None


@dataclass
class Scenario:
    name: str
    met: MetSpec
    sources: list
    start: int
    end: int
    dt: int
    out_shape: tuple
    outheights: list
    key: tuple = (42, 0)
    dry_velocity: float = 0.002
    wet_a: float = 1.0e-4
    wet_b: float = 0.8
    capacity: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def n_steps(self) -> int:
        # has_remaining_steps is inclusive (simulation/timeloop.rs:832-834)
        return (self.end - self.start) // self.dt + 1


def level_heights(nz: int, top_m: float) -> np.ndarray:
    """Terrain-following levels stretched quadratically to `top_m` (no terrain:
    heights are the same in every column)."""
    k = np.arange(1, nz + 1, dtype=np.float64)
    return (top_m * (k / nz) ** 2).astype(np.float32)


def velocity_scale(spec: MetSpec) -> tuple:
    """One global metres->grid factor at the domain-centre latitude
    (VelocityToGridScale, src/physics/advection.rs:36-41, built as in
    src/bin/fortran-validation.rs:123-138)."""
    lat_c = spec.ylat0 + 0.5 * (spec.ny - 1) * spec.dy_deg
    dx_m = R_EARTH * math.cos(math.radians(lat_c)) * math.radians(spec.dx_deg)
    dy_m = R_EARTH * math.radians(spec.dy_deg)
    return (float(np.float32(1.0 / dx_m)), float(np.float32(1.0 / dy_m)), 1.0)


def _smooth_normal(rng, shape, mean, std, sigma_cells):
    from scipy.ndimage import gaussian_filter

    a = rng.standard_normal(shape)
    a = gaussian_filter(a, sigma=(sigma_cells, sigma_cells, 0), mode="wrap")
    a = (a - a.mean()) / max(a.std(), 1e-12)
    return (mean + std * a).astype(np.float32)


def make_frames(spec: MetSpec):
    """Returns a list of n_frames dicts with u, v, w of shape (nx, ny, nz)
    in the reference layout ((ix*ny)+iy)*nz+iz, and the surface cell
    records of each frame."""
    rng = np.random.default_rng(1_000 + spec.seed)
    shape = (spec.nx, spec.ny, spec.nz)
    pbl_h = rng.uniform(300.0, 1500.0, (spec.nx, spec.ny)).astype(np.float32)
    ustar = rng.uniform(0.1, 0.6, (spec.nx, spec.ny)).astype(np.float32)
    oli = rng.normal(0.0, 0.01, (spec.nx, spec.ny)).astype(np.float32)
    frames = []
    for f in range(spec.n_frames):
        u = _smooth_normal(rng, shape, 5.0, 3.0, 3.0)
        v = _smooth_normal(rng, shape, 5.0, 3.0, 3.0)
        w = rng.normal(0.0, 0.05, shape).astype(np.float32)
        # PBL inputs vary slowly between frames (+-10 %)
        h_f = (pbl_h * rng.uniform(0.9, 1.1, pbl_h.shape)).astype(np.float32)
        us_f = (ustar * rng.uniform(0.9, 1.1, ustar.shape)).astype(np.float32)
        oli_f = (oli * rng.uniform(0.9, 1.1, oli.shape)).astype(np.float32)
        frames.append({"u": u, "v": v, "w": w, "surface": surface_cells(spec, u, v, h_f, us_f, oli_f)})
    return frames


def surface_cells(spec: MetSpec, u, v, hmix, ustar, oli) -> np.ndarray:
    """fpg_surface_cell records with met-provided u*, 1/L and h, and the
    sensible heat flux that gives the same L through the flux formula
    (pbl_diagnostics.wgsl:168-195: L = -(rho cp T u*^3) / (kappa g H))."""
    n = spec.nx * spec.ny
    cells = np.zeros(n, SURFACE_DTYPE)
    t2m = np.float32(288.15)                     # sea level; 6.5 K/km lapse aloft
    sp = np.float32(101_325.0)
    rho = sp / (np.float32(287.05) * t2m)
    cells["surface_pressure_pa"] = sp
    cells["temperature_2m_k"] = t2m
    cells["u10_ms"] = u[:, :, 0].reshape(n)
    cells["v10_ms"] = v[:, :, 0].reshape(n)
    us = ustar.reshape(n).astype(np.float32)
    cells["surface_stress_n_m2"] = (rho * us * us).astype(np.float32)
    shf = -(rho * np.float32(1004.6) * t2m * us ** 3) * oli.reshape(n) / (np.float32(0.4) * np.float32(9.81))
    cells["sensible_heat_flux_w_m2"] = shf.astype(np.float32)
    cells["solar_radiation_w_m2"] = np.float32(250.0)
    cells["mixing_height_m"] = hmix.reshape(n)
    cells["friction_velocity_ms"] = us
    cells["inv_obukhov_length_per_m"] = oli.reshape(n)
    return cells


def precipitation(spec: MetSpec, frame: int):
    """Lognormal(-1, 1) mm/h on a random 30 % of cells (large-scale), zero
    elsewhere; no convective part; cloud cover 1."""
    rng = np.random.default_rng(5_000 + 31 * spec.seed + frame)
    n = spec.nx * spec.ny
    lsp = np.zeros(n, np.float32)
    on = rng.random(n) < 0.30
    lsp[on] = rng.lognormal(-1.0, 1.0, int(on.sum())).astype(np.float32)
    return lsp


EPOCH_2024 = 1_704_067_200  # 2024-01-01 00:00:00 UTC


def config0() -> Scenario:
    """100 k particles, one point release of 1 kg spread over 1 h at 50 m AGL;
    met 90x60 (0.5 deg) x 20 levels to 15 km; 2 frames 3 h apart cycled for
    24 h; dt 900 s (97 inclusive steps); output 90x60x3 (100, 500, 1000 m)."""
    met = MetSpec(nx=90, ny=60, nz=20, dx_deg=0.5, dy_deg=0.5, xlon0=-10.0, ylat0=35.0, n_frames=2, seed=0)
    t0 = EPOCH_2024
    src = Source(lon=met.xlon0 + 15.25, lat=met.ylat0 + 15.25, z_min=50.0, z_max=50.0, mass_kg=1.0,
                 particle_count=100_000, start=t0, end=t0 + 3600)
    return Scenario("config0", met, [src], start=t0, end=t0 + 24 * 3600, dt=900, out_shape=(90, 60, 3),
                    outheights=[100.0, 500.0, 1000.0], capacity=100_000)


def config1(particles: int = 10_000_000) -> Scenario:
    """10 M particles from 8 point sources (random locations, heights
    U(10, 300) m, 1 kg/h each) released over 48 h; met 360x180 (1 deg) x 60
    levels, 9 frames 3 h apart (cycled); wet scavenging on; output 360x180x5."""
    met = MetSpec(nx=360, ny=180, nz=60, dx_deg=1.0, dy_deg=1.0, xlon0=-180.0, ylat0=-89.5, n_frames=9, seed=1,
                  wet=True)
    rng = np.random.default_rng(77)
    t0 = EPOCH_2024
    per = particles // 8
    sources = []
    for s in range(8):
        lon = float(rng.uniform(-150.0, 150.0))
        lat = float(rng.uniform(-60.0, 60.0))
        z = float(rng.uniform(10.0, 300.0))
        sources.append(Source(lon=lon, lat=lat, z_min=z, z_max=z, mass_kg=48.0,
                              particle_count=per + (1 if s < particles - 8 * per else 0),
                              start=t0, end=t0 + 48 * 3600))
    return Scenario("config1", met, sources, start=t0, end=t0 + 48 * 3600, dt=900, out_shape=(360, 180, 5),
                    outheights=[100.0, 500.0, 1000.0, 2000.0, 5000.0], capacity=particles)


def bracket_frames(scn: Scenario, t: int):
    """(frame index t0, frame index t1, time t0, time t1) of the bracket that
    holds t; frames cycle with period n_frames."""
    fs = scn.met.frame_seconds
    k = (t - scn.start) // fs
    if t - scn.start == k * fs and k > 0:
        k -= 1  # at a frame time, stay in the bracket that ends there
    ta = scn.start + k * fs
    n = scn.met.n_frames
    return int(k % n), int((k + 1) % n), ta, ta + fs


def particles_at_sources(scn: Scenario, n: int, seed: int = 3) -> np.ndarray:
    """n active particle records scattered in the boxes around the sources
    (used where a test needs an already-spread population)."""
    rng = np.random.default_rng(seed)
    spec = scn.met
    rec = np.zeros(n, PARTICLE_DTYPE)
    # consecutive slots belong to one source, as the release manager fills
    # them (release/mod.rs:103-146)
    src_idx = np.sort(rng.integers(0, len(scn.sources), n))
    lon = np.array([s.lon for s in scn.sources])[src_idx] + rng.normal(0, 3.0 * spec.dx_deg, n)
    lat = np.array([s.lat for s in scn.sources])[src_idx] + rng.normal(0, 3.0 * spec.dy_deg, n)
    x = np.clip((lon - spec.xlon0) / spec.dx_deg, 0, spec.nx - 1.001)
    y = np.clip((lat - spec.ylat0) / spec.dy_deg, 0, spec.ny - 1.001)
    fx, fy = np.floor(x), np.floor(y)
    rec["cell_x"] = fx.astype(np.int32)
    rec["cell_y"] = fy.astype(np.int32)
    rec["pos_x"] = (x - fx).astype(np.float32)
    rec["pos_y"] = (y - fy).astype(np.float32)
    rec["pos_z"] = rng.uniform(1.0, 2500.0, n).astype(np.float32)
    rec["flags"] = 1
    rec["mass"][:, 0] = np.float32(1.0 / n)
    rec["turb_u"] = rng.normal(0, 0.5, n).astype(np.float32)
    rec["turb_v"] = rng.normal(0, 0.5, n).astype(np.float32)
    rec["turb_w"] = rng.normal(0, 0.3, n).astype(np.float32)
    return rec


@dataclass
class Ensemble:
    """Many independent release scenarios on one met set (the batched run)."""

    name: str
    met: MetSpec
    sources: list          # one Source per scenario
    keys: list             # (k0, k1) per scenario
    start: int
    end: int
    dt: int
    out_shape: tuple
    outheights: list
    dry_velocity: float = 0.002
    wet_a: float = 1.0e-4
    wet_b: float = 0.8

    @property
    def n_steps(self) -> int:
        return (self.end - self.start) // self.dt + 1

    @property
    def total_particles(self) -> int:
        return sum(s.particle_count for s in self.sources)

    def scenario(self, s: int) -> Scenario:
        """Scenario s alone, as a plain single-release run."""
        src = self.sources[s]
        return Scenario(f"{self.name}[{s}]", self.met, [src], start=self.start, end=self.end, dt=self.dt,
                        out_shape=self.out_shape, outheights=self.outheights, key=self.keys[s],
                        dry_velocity=self.dry_velocity, wet_a=self.wet_a, wet_b=self.wet_b,
                        capacity=src.particle_count)


def config2(n_scenarios: int = 256, lo: int = 10_000, hi: int = 1_000_000, hours: int = 24,
            met: MetSpec | None = None, seed: int = 2) -> Ensemble:
    """n_scenarios point releases with particle counts log-uniform in
    [lo, hi] (about 55 M for 256 in [10 k, 1 M]), each with its own source
    location, height U(10, 300) m, start time (a step boundary in the first
    half of the run), 6 h release window, 1 kg and Philox key; met
    180x90 (2 deg) x 40 levels, 9 frames 3 h apart, wet scavenging on;
    per-scenario output 180x90x3."""
    if met is None:
        met = MetSpec(nx=180, ny=90, nz=40, dx_deg=2.0, dy_deg=2.0, xlon0=-179.0, ylat0=-89.0, n_frames=9,
                      seed=2, wet=True)
    rng = np.random.default_rng(200 + seed)
    t0 = EPOCH_2024
    dt = 900
    end = t0 + hours * 3600
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), n_scenarios)).astype(np.int64)
    lon_span = (met.nx - 1) * met.dx_deg
    lat_span = (met.ny - 1) * met.dy_deg
    sources, keys = [], []
    half_steps = max((end - t0) // dt // 2, 1)
    for s in range(n_scenarios):
        lon = float(met.xlon0 + rng.uniform(0.1, 0.9) * lon_span)
        lat = float(met.ylat0 + rng.uniform(0.2, 0.8) * lat_span)
        z = float(rng.uniform(10.0, 300.0))
        start = int(t0 + dt * int(rng.integers(0, half_steps)))
        rel_end = min(start + 6 * 3600, end)
        sources.append(Source(lon=lon, lat=lat, z_min=z, z_max=z, mass_kg=1.0, particle_count=int(counts[s]),
                              start=start, end=rel_end))
        keys.append((int(rng.integers(0, 2**32)), s))
    return Ensemble("config2", met, sources, keys, start=t0, end=end, dt=dt, out_shape=(met.nx, met.ny, 3),
                    outheights=[100.0, 500.0, 1000.0])


@dataclass
class Inversion:
    """A source-inversion problem: sources (one batch scenario each, own key),
    receptors (cells of the lowest layer), observations."""

    name: str
    ensemble: Ensemble         # sources as scenarios, with their true masses
    receptors: list            # (instance, i, j)
    instance: list             # instance of each source
    sample_every: int = 12
    receptor_top_m: float = 100.0
    receptor_ramp_m: float = 20.0
    checkpoint_every: int = 8
    tape_tail_windows: int = 0  # last windows taped in the forward (not recomputed)


def config3(n_particles: int = 1_000_000, n_sources: int = 16, n_receptors: int = 200, hours: int = 24,
            met: MetSpec | None = None, seed: int = 3, smooth: bool = False) -> Inversion:
    """Source inversion on the configuration-0 met (90x60 at 0.5 deg x 20
    levels, 2 frames 3 h apart, cycled): n_sources point sources at heights
    U(10, 300) m with 1 kg each, released over 6 h from a step in the first
    half of the run, n_particles in all (equal shares), their own Philox
    keys; n_receptors distinct random cells of the lowest layer (0-100 m),
    sampled every 3 h; dt 900 s.  smooth=True makes the PBL inputs uniform
    in space and switches deposition off, so the forward map has no
    discontinuity in position (for finite-difference checks)."""
    if met is None:
        met = MetSpec(nx=90, ny=60, nz=20, dx_deg=0.5, dy_deg=0.5, xlon0=-10.0, ylat0=35.0, n_frames=2, seed=0)
    rng = np.random.default_rng(300 + seed)
    t0 = EPOCH_2024
    dt = 900
    end = t0 + hours * 3600
    per = n_particles // n_sources
    sources, keys = [], []
    half_steps = max((end - t0) // dt // 2, 1)
    lon_span = (met.nx - 1) * met.dx_deg
    lat_span = (met.ny - 1) * met.dy_deg
    for s in range(n_sources):
        lon = float(met.xlon0 + rng.uniform(0.25, 0.75) * lon_span)
        lat = float(met.ylat0 + rng.uniform(0.25, 0.75) * lat_span)
        z = float(rng.uniform(10.0, 300.0))
        start = int(t0 + dt * int(rng.integers(0, half_steps)))
        sources.append(Source(lon=lon, lat=lat, z_min=z, z_max=z, mass_kg=1.0,
                              particle_count=per + (1 if s < n_particles - per * n_sources else 0),
                              start=start, end=min(start + 6 * 3600, end)))
        keys.append((int(rng.integers(0, 2**32)), 1000 + s))
    cells = rng.choice(met.nx * met.ny, size=n_receptors, replace=False)
    receptors = [(0, int(c // met.ny), int(c % met.ny)) for c in cells]
    ens = Ensemble("config3", met, sources, keys, start=t0, end=end, dt=dt, out_shape=(met.nx, met.ny, 1),
                   outheights=[100.0], dry_velocity=0.0 if smooth else 0.002)
    inv = Inversion("config3", ens, receptors, [0] * n_sources)
    inv.smooth = smooth
    return inv


def make_frames_uniform_pbl(spec: MetSpec):
    """make_frames with every surface cell replaced by the first cell's
    values (spatially uniform PBL inputs)."""
    frames = make_frames(spec)
    for f in frames:
        f["surface"][:] = f["surface"][0]
    return frames


def config4(n_instances: int = 64, lo: int = 50_000, hi: int = 2_000_000, hours: int = 72, sources_per: int = 8,
            receptors_per: int = 100, met: MetSpec | None = None, seed: int = 4) -> Inversion:
    """n_instances independent source inversions in one batch: particle
    counts per instance log-uniform in [lo, hi] (about 34 M for 64 in
    [50 k, 2 M]), split over sources_per point sources (heights U(10, 300)
    m, 6 h releases from a step in the first half, own Philox keys), and
    receptors_per distinct receptor cells per instance; met 180x90 (2 deg) x
    40 levels, 9 frames 3 h apart, wet scavenging on; 72 h (289 steps) at
    dt 900 s; checkpoints every 8 steps."""
    if met is None:
        met = MetSpec(nx=180, ny=90, nz=40, dx_deg=2.0, dy_deg=2.0, xlon0=-179.0, ylat0=-89.0, n_frames=9,
                      seed=2, wet=True)
    rng = np.random.default_rng(400 + seed)
    t0 = EPOCH_2024
    dt = 900
    end = t0 + hours * 3600
    half_steps = max((end - t0) // dt // 2, 1)
    lon_span = (met.nx - 1) * met.dx_deg
    lat_span = (met.ny - 1) * met.dy_deg
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), n_instances)).astype(np.int64)
    sources, keys, instance, receptors = [], [], [], []
    for n in range(n_instances):
        per = int(counts[n]) // sources_per
        for s in range(sources_per):
            lon = float(met.xlon0 + rng.uniform(0.1, 0.9) * lon_span)
            lat = float(met.ylat0 + rng.uniform(0.2, 0.8) * lat_span)
            z = float(rng.uniform(10.0, 300.0))
            start = int(t0 + dt * int(rng.integers(0, half_steps)))
            sources.append(Source(lon=lon, lat=lat, z_min=z, z_max=z, mass_kg=1.0, particle_count=max(per, 1),
                                  start=start, end=min(start + 6 * 3600, end)))
            keys.append((int(rng.integers(0, 2**32)), 100_000 + n * sources_per + s))
            instance.append(n)
        cells = rng.choice(met.nx * met.ny, size=receptors_per, replace=False)
        receptors += [(n, int(c // met.ny), int(c % met.ny)) for c in cells]
    ens = Ensemble("config4", met, sources, keys, start=t0, end=end, dt=dt, out_shape=(met.nx, met.ny, 1),
                   outheights=[100.0])
    inv = Inversion("config4", ens, receptors, instance, checkpoint_every=8)
    inv.smooth = False
    return inv
