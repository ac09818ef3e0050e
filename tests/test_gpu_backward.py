"""Backward (receptor) mode behind the C ABI (fpg_backward_*).

* The reference's own backward tests, restated: receptor release at the
  start time, alpha sequence 1, 0.5, 0 over a backward bracket, drift
  against the wind (tests/backward_timeloop.rs:48-158); a forward run from a
  source and a backward run from the receptor it reaches each collect
  exactly the released particle and its mass
  (tests/integration/source_receptor_consistency.rs:281-364).
* Against the oracle's backward loop on the configuration-0 met: per-step
  reports (released count, alpha, Philox counter) bit-exact, particle state
  within the step tolerance, and source collections equal to a host
  recount of the device's own particle positions (counts exact, double
  masses to rounding).
* The reference's validation errors.
"""
import numpy as np
import pytest

from flexpart_gpu import synthetic
from flexpart_gpu._lib import FpgError
from flexpart_gpu.records import SURFACE_DTYPE, GridDomain, MetBracket, ReceptorRelease, SourceRegion
from helpers import assert_parity

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")
tl = pytest.importorskip("flexpart_gpu.timeloop")

T0 = 1_704_067_200  # 20240101000000


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _uniform_met(nx=64, ny=64, nz=16, u=1.0):
    """The reference tests' met: uniform wind, levels at 0..nz-1 m, neutral
    surface with a 1000 m mixing height (backward_timeloop.rs:11-46)."""
    wind = {"u": np.full(nx * ny * nz, u, np.float32), "v": np.zeros(nx * ny * nz, np.float32),
            "w": np.zeros(nx * ny * nz, np.float32)}
    s = np.zeros(nx * ny, SURFACE_DTYPE)
    s["surface_pressure_pa"] = 101_325.0
    s["u10_ms"] = 1.0
    s["temperature_2m_k"] = 290.0
    s["mixing_height_m"] = 1_000.0
    return wind, s, np.arange(nz, dtype=np.float32)


def _bracket(wind, surf, t0, t1):
    return MetBracket(wind["u"].ctypes.data, wind["v"].ctypes.data, wind["w"].ctypes.data, wind["u"].ctypes.data,
                      wind["v"].ctypes.data, wind["w"].ctypes.data, surf.ctypes.data, surf.ctypes.data, t0, t1)


def test_backward_receptor_release_alpha_and_drift(ctx):
    wind, surf, heights = _uniform_met()
    cfg = tl.backward_config(start_seconds=T0 + 2, end_seconds=T0, timestep_seconds=1, clamp_time_bounds=0)
    grid = GridDomain(0.0, 0.0, 1.0, 1.0, 64, 64)
    drv = tl.BackwardDriver(ctx, cfg, [ReceptorRelease(10.0, 5.0, 1.0, 1, 1.0)],
                            [SourceRegion(6.9, 7.1, 4.9, 5.1, 0.0, 5.0)], grid, 8, (64, 64, 16), heights)
    met = _bracket(wind, surf, T0, T0 + 2)
    reports = []
    while drv.has_remaining_steps:
        reports.append(drv.run_timestep(met, tl.uniform_forcing()))
    assert len(reports) == 3
    assert [r.released_count for r, _ in reports] == [1, 0, 0]
    assert np.allclose([r.interpolation_alpha for r, _ in reports], [1.0, 0.5, 0.0], atol=1e-6)
    assert [r.simulation_time_seconds for r, _ in reports] == [T0 + 2, T0 + 1, T0]
    p = drv.particles.download(0, 1)[0]
    gx, gy = p["cell_x"] + float(p["pos_x"]), p["cell_y"] + float(p["pos_y"])
    assert p["flags"] & 1
    assert 4.0 < gx < 10.0, gx
    assert abs(gy - 5.0) < 2.0, gy
    assert abs(float(p["mass"][0]) - 1.0) < 1e-6
    assert len(reports[-1][1]) == 1
    with pytest.raises(FpgError):
        drv.run_timestep(met, tl.uniform_forcing())


def test_source_receptor_consistency(ctx):
    """Forward from a source at (7, 5, 1 m) reaches the receptor box around
    (10, 5); backward from a receptor at (10, 5, 1 m) reaches the source box
    around (7, 5); each collects the one particle and its 1 kg."""
    wind, surf, heights = _uniform_met()
    grid = GridDomain(0.0, 0.0, 1.0, 1.0, 64, 64)
    met = _bracket(wind, surf, T0, T0 + 2)
    fcfg = tl.default_config(start_seconds=T0, end_seconds=T0 + 2, timestep_seconds=1, clamp_time_bounds=0)
    from flexpart_gpu.records import Release

    fwd = tl.ForwardDriver(ctx, fcfg, [Release(T0, T0, 7.0, 7.0, 5.0, 5.0, 1.0, 1.0, 1.0, 1)], grid, 8,
                           (64, 64, 16), heights)
    n = 0
    while fwd.has_remaining_steps:
        fwd.run_timestep(met, tl.uniform_forcing())
        n += 1
    assert n == 3
    rec = fwd.particles.download()
    act = (rec["flags"] & 1) != 0
    lon = rec["cell_x"].astype(np.float64) + rec["pos_x"].astype(np.float64)
    lat = rec["cell_y"].astype(np.float64) + rec["pos_y"].astype(np.float64)
    z = rec["pos_z"].astype(np.float64)
    inside = act & (lon >= 8.0) & (lon <= 12.0) & (lat >= 3.0) & (lat <= 7.0) & (z >= 0.0) & (z <= 16.0)
    fwd_hits, fwd_mass = int(inside.sum()), float(rec["mass"][inside, 0].sum())

    bcfg = tl.backward_config(start_seconds=T0 + 2, end_seconds=T0, timestep_seconds=1, clamp_time_bounds=0)
    bwd = tl.BackwardDriver(ctx, bcfg, [ReceptorRelease(10.0, 5.0, 1.0, 1, 1.0)],
                            [SourceRegion(5.0, 9.0, 3.0, 7.0, 0.0, 16.0)], grid, 8, (64, 64, 16), heights)
    last = None
    while bwd.has_remaining_steps:
        last = bwd.run_timestep(met, tl.uniform_forcing())
    hits, mass32, mass64 = last[1][0]
    assert fwd_hits == 1 and hits == 1
    assert abs(fwd_mass - 1.0) < 1e-6 and abs(mass32 - 1.0) < 1e-6
    assert abs(fwd_mass - mass32) <= 1e-6


def _config0_backward(hours=6, per_receptor=5_000):
    scn = synthetic.config0()
    spec = scn.met
    start = scn.start + 24 * 3600
    end = start - hours * 3600
    lons = [spec.xlon0 + 10.25, spec.xlon0 + 20.75, spec.xlon0 + 30.5, spec.xlon0 + 15.0]
    lats = [spec.ylat0 + 12.5, spec.ylat0 + 18.25, spec.ylat0 + 10.0, spec.ylat0 + 22.0]
    receptors = [ReceptorRelease(lo, la, 30.0 + 40.0 * k, per_receptor, 0.5 + k) for k, (lo, la) in
                 enumerate(zip(lons, lats))]
    regions = [SourceRegion(spec.xlon0 + 5.0, spec.xlon0 + 12.0, spec.ylat0 + 8.0, spec.ylat0 + 16.0, 0.0, 2000.0),
               SourceRegion(spec.xlon0 + 14.0, spec.xlon0 + 26.0, spec.ylat0 + 14.0, spec.ylat0 + 24.0, 0.0, 500.0),
               SourceRegion(spec.xlon0, spec.xlon0 + 44.5, spec.ylat0, spec.ylat0 + 29.5, 0.0, 15000.0)]
    # the oracle's scenario: receptors as point sources released at the start time
    oscn = synthetic.Scenario("backward", spec, [synthetic.Source(r.lon, r.lat, r.z_m, r.z_m, r.mass_kg,
                                                                  r.particle_count, start, start) for r in receptors],
                              start=start, end=end, dt=900, out_shape=scn.out_shape, outheights=scn.outheights,
                              key=(42, 0), capacity=per_receptor * len(receptors))
    return scn, oscn, receptors, regions


def test_backward_steps_match_the_oracle_backward_loop(ctx):
    from oracle.forward import OracleBackward

    scn, oscn, receptors, regions = _config0_backward()
    spec = scn.met
    frames = synthetic.make_frames(spec)
    src = tl.BracketSource(scn, frames)     # frames anchored at the configuration's start

    def bracket(t):
        fa, fb, ta, tb = synthetic.bracket_frames(scn, t)
        return frames[fa], frames[fb], ta, tb

    xs, ys, zs = synthetic.velocity_scale(spec)
    cfg = tl.backward_config(start_seconds=oscn.start, end_seconds=oscn.end, timestep_seconds=900,
                             x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, philox_key=(42, 0))
    cap = oscn.capacity
    drv = tl.BackwardDriver(ctx, cfg, receptors, regions, tl.scenario_domain(scn), cap, (spec.nx, spec.ny, spec.nz),
                            synthetic.level_heights(spec.nz, spec.top_m))
    reg = [{k: getattr(r, k) for k, _ in r._fields_} for r in regions]
    ob = OracleBackward(oscn, cap, frames, reg, bracket)
    ob64 = OracleBackward(oscn, cap, frames, reg, bracket, dtype=np.float64)
    forcing = tl.uniform_forcing(dry_velocity=0.002)
    k = 0
    while drv.has_remaining_steps:
        z_prev = ob.records()["pos_z"]
        rep, col = drv.run_timestep(src.at(drv.current_time_seconds), forcing)
        orep = ob.run_timestep({"dry_velocity": 0.002})
        ob64.run_timestep({"dry_velocity": 0.002})
        assert rep.released_count == orep["released"]
        assert rep.interpolation_alpha == np.float32(orep["alpha"])
        assert list(rep.next_philox_counter) == orep["counter"]
        assert rep.simulation_time_seconds == orep["time"]
        g = drv.particles.download()
        if k < 3:
            o = ob.records()
            z_in = np.where(z_prev == 0.0, o["pos_z"], z_prev)
            assert_parity(g, ob.state, z_in, ob64.state, f"backward step {k}")
        # the device's collections recounted on the host from its own particles
        act = (g["flags"] & 1) != 0
        lon = spec.xlon0 + (g["cell_x"].astype(np.float64) + g["pos_x"].astype(np.float64)) * spec.dx_deg
        lat = spec.ylat0 + (g["cell_y"].astype(np.float64) + g["pos_y"].astype(np.float64)) * spec.dy_deg
        z = g["pos_z"].astype(np.float64)
        for (hits, m32, m64), r, (ohits, _, om64) in zip(col, regions, orep["collections"]):
            inside = act & (lon >= r.lon_min) & (lon <= r.lon_max) & (lat >= r.lat_min) & (lat <= r.lat_max) & \
                (z >= r.z_min_m) & (z <= r.z_max_m)
            assert hits == int(inside.sum())
            host64 = float(g["mass"][inside, 0].astype(np.float64).sum())
            assert abs(m64 - host64) <= 1e-12 * max(abs(host64), 1e-30)
            assert m32 == np.float32(m64)
            # against the oracle's own positions: boundary flips only
            assert abs(hits - ohits) <= max(2, ohits // 200)
        k += 1
    assert k == 25
    assert col[2][0] == cap  # the whole-domain region holds every particle


def test_backward_validation_errors(ctx):
    wind, surf, heights = _uniform_met()
    grid = GridDomain(0.0, 0.0, 1.0, 1.0, 64, 64)
    rec = [ReceptorRelease(10.0, 5.0, 1.0, 1, 1.0)]
    reg = [SourceRegion(6.9, 7.1, 4.9, 5.1, 0.0, 5.0)]

    def status(cfg, r=rec, g=reg):
        with pytest.raises(FpgError) as e:
            tl.BackwardDriver(ctx, cfg, r, g, grid, 8, (64, 64, 16), heights)
        return e.value.status

    assert status(tl.backward_config(start_seconds=T0, end_seconds=T0 + 2)) == -19
    assert status(tl.backward_config(start_seconds=T0 + 2, end_seconds=T0), r=[]) == -20
    assert status(tl.backward_config(start_seconds=T0 + 2, end_seconds=T0),
                  r=[ReceptorRelease(190.0, 5.0, 1.0, 1, 1.0)]) == -21
    assert status(tl.backward_config(start_seconds=T0 + 2, end_seconds=T0),
                  r=[ReceptorRelease(10.0, 5.0, 1.0, 0, 1.0)]) == -21
    assert status(tl.backward_config(start_seconds=T0 + 2, end_seconds=T0),
                  g=[SourceRegion(7.1, 6.9, 4.9, 5.1, 0.0, 5.0)]) == -22
    assert status(tl.backward_config(start_seconds=T0 + 2, end_seconds=T0, timestep_seconds=0)) == -2


def test_backward_separated_passes_give_the_fused_bits(ctx):
    """The reference's backward driver always runs the separated Hanna,
    Langevin and deposition passes (timeloop.rs:1433-1437); with them the
    device's particles and source collections equal the fused kernel's, bit
    for bit, after every step."""
    scn, oscn, receptors, regions = _config0_backward(hours=3, per_receptor=2_000)
    spec = scn.met
    frames = synthetic.make_frames(spec)
    src = tl.BracketSource(scn, frames)
    xs, ys, zs = synthetic.velocity_scale(spec)
    cfg = tl.backward_config(start_seconds=oscn.start, end_seconds=oscn.end, timestep_seconds=900,
                             x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, philox_key=(42, 0))
    drivers = [tl.BackwardDriver(ctx, cfg, receptors, regions, tl.scenario_domain(scn), oscn.capacity,
                                 (spec.nx, spec.ny, spec.nz), synthetic.level_heights(spec.nz, spec.top_m))
               for _ in range(2)]
    drivers[1].set_validation_mode(True)
    forcing = tl.uniform_forcing(dry_velocity=0.002)
    steps = 0
    while drivers[0].has_remaining_steps:
        (ra, ca), (rb, cb) = (d.run_timestep(src.at(d.current_time_seconds), forcing) for d in drivers)
        assert list(ra.next_philox_counter) == list(rb.next_philox_counter) and ca == cb
        assert drivers[0].particles.download().tobytes() == drivers[1].particles.download().tobytes(), steps
        steps += 1
    assert steps == 13
