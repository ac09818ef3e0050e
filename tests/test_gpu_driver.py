"""The forward time loop behind the C ABI (fpg_forward_*) against the oracle's
forward loop: per-step reports (released counts, alpha, Philox counter,
active count) bit-exact, particle state within the step tolerance on the
first steps, and after the full 24 h run of the 100 k-particle configuration
the gridded mass per cell within 1e-4 of the released mass (1 kg)."""
import numpy as np
import pytest

from flexpart_gpu import synthetic
from helpers import assert_parity
from oracle.forward import OracleForward

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")
tl = pytest.importorskip("flexpart_gpu.timeloop")


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _small(particles=20_000, hours=6):
    scn = synthetic.config0()
    scn.sources[0].particle_count = particles
    scn.capacity = particles
    scn.end = scn.start + hours * 3600
    return scn


def _driver(ctx, scn, **kw):
    cfg = tl.scenario_config(scn, **kw)
    return tl.ForwardDriver(ctx, cfg, tl.scenario_releases(scn), tl.scenario_domain(scn), scn.capacity,
                            (scn.met.nx, scn.met.ny, scn.met.nz),
                            synthetic.level_heights(scn.met.nz, scn.met.top_m))


def _check_report(rep, orep):
    assert rep.released_count == orep["released"]
    assert rep.interpolation_alpha == np.float32(orep["alpha"])
    assert list(rep.next_philox_counter) == orep["counter"]
    assert rep.active_particle_count == orep["active"]


@pytest.mark.parametrize("mode", ["plain", "compaction", "sort"])
def test_driver_steps_match_oracle_loop(ctx, mode):
    scn = _small()
    frames = synthetic.make_frames(scn.met)
    kw = {"use_compaction": 1} if mode == "compaction" else {"sort_interval_steps": 3} if mode == "sort" else {}
    okw = {"use_compaction": True} if mode == "compaction" else {"sort_interval": 3} if mode == "sort" else {}
    drv = _driver(ctx, scn, **kw)
    fw = OracleForward(scn, scn.capacity, frames, **okw)
    fw64 = OracleForward(scn, scn.capacity, frames, dtype=np.float64, **okw)
    src = tl.BracketSource(scn, frames)
    forcing = tl.uniform_forcing(dry_velocity=0.002)
    for k in range(8):
        z_prev = fw.records()["pos_z"]
        rep = drv.run_timestep(src.at(drv.current_time_seconds), forcing)
        orep = fw.run_timestep({"dry_velocity": 0.002})
        fw64.run_timestep({"dry_velocity": 0.002})
        _check_report(rep, orep)
        if k < 3:
            g = drv.particles.download()
            o = fw.records()
            # heights at the step start (release height for particles released this step)
            z_in = np.where(z_prev == 0.0, o["pos_z"], z_prev)
            assert_parity(g, fw.state, z_in, fw64.state, f"{mode} step {k}")
            assert np.array_equal(g["release_point"], o["release_point"])
            assert np.array_equal(g["time"], o["time"])


def test_full_24h_run_gridded_mass_within_1e4_of_released(ctx):
    scn = synthetic.config0()
    frames = synthetic.make_frames(scn.met)
    drv = _driver(ctx, scn)
    src = tl.BracketSource(scn, frames)
    forcing = tl.uniform_forcing(dry_velocity=scn.dry_velocity)
    fw = OracleForward(scn, scn.capacity, frames)
    fw64 = OracleForward(scn, scn.capacity, frames, dtype=np.float64)
    steps = 0
    while drv.has_remaining_steps:
        rep = drv.run_timestep(src.at(drv.current_time_seconds), forcing)
        orep = fw.run_timestep({"dry_velocity": scn.dry_velocity})
        fw64.run_timestep({"dry_velocity": scn.dry_velocity})
        _check_report(rep, orep)
        steps += 1
    drv.finalize()
    assert steps == 97 and not fw.has_remaining_steps
    grid = api.Grid(ctx, *scn.out_shape)
    counts, mass, kg = drv.accumulate_concentration_grid(grid, 0, 1e6, scn.outheights)
    oc, om, _ = fw.grid()
    oc64, om64, _ = fw64.grid()
    released = sum(s.mass_kg for s in scn.sources)
    d_gpu = np.abs(mass.astype(np.int64) - om.astype(np.int64)) / 1e6
    d_fp32 = np.abs(om.astype(np.int64) - om64.astype(np.int64)) / 1e6
    d_gpu64 = np.abs(mass.astype(np.int64) - om64.astype(np.int64)) / 1e6
    print(f"24 h: max |mass_gpu - mass_oracle32| = {d_gpu.max():.2e} kg, vs FP64 {d_gpu64.max():.2e} kg; "
          f"oracle32 vs FP64 {d_fp32.max():.2e} kg; counts differ by at most "
          f"{np.abs(counts.astype(np.int64) - oc.astype(np.int64)).max()}")
    assert counts.sum() == oc.sum() == 100_000
    assert d_gpu.max() <= 1e-4 * released
    assert d_gpu64.max() <= 1e-4 * released


def test_driver_errors(ctx):
    scn = _small(1000, 1)
    with pytest.raises(api._lib.FpgError) as e:
        tl.ForwardDriver(ctx, tl.scenario_config(scn, start_seconds=scn.end + 1), tl.scenario_releases(scn),
                         tl.scenario_domain(scn), 1000, (scn.met.nx, scn.met.ny, scn.met.nz))
    assert e.value.status == -18     # InvalidTimeRange (timeloop.rs:1935)
    with pytest.raises(api._lib.FpgError) as e:
        tl.ForwardDriver(ctx, tl.scenario_config(scn, timestep_seconds=0), tl.scenario_releases(scn),
                         tl.scenario_domain(scn), 1000, (scn.met.nx, scn.met.ny, scn.met.nz))
    assert e.value.status == -2      # InvalidTimestep
    drv = _driver(ctx, scn)
    frames = synthetic.make_frames(scn.met)
    src = tl.BracketSource(scn, frames)
    while drv.has_remaining_steps:
        drv.run_timestep(src.at(drv.current_time_seconds), tl.uniform_forcing())
    with pytest.raises(api._lib.FpgError) as e:
        drv.run_timestep(src.at(scn.end), tl.uniform_forcing())
    assert e.value.status == -14     # SimulationComplete (timeloop.rs:921)
    small = _small(1000, 1)
    small.capacity = 500             # the release overflows the store
    drv2 = _driver(ctx, small)
    with pytest.raises(api._lib.FpgError) as e:
        for _ in range(5):
            drv2.run_timestep(src.at(drv2.current_time_seconds), tl.uniform_forcing())
    assert e.value.status == -9      # StoreFull (particles/mod.rs:516)


def _run_with_ring(ctx, scn, frames, mode):
    """24 h over 3 h brackets; mode "host": frames from the bracket's host
    pointers; "ring": every frame prefetched a bracket ahead; "mixed": only
    the frames of every other bracket prefetched, so half the brackets miss
    the ring and fall back to the host pointers."""
    drv = _driver(ctx, scn)
    src = tl.BracketSource(scn, frames)
    forcing = tl.uniform_forcing(dry_velocity=scn.dry_velocity)
    fs = scn.met.frame_seconds
    if mode != "host":
        drv.enable_met_ring(3)
    prefetched = set()
    dev = None
    if mode == "device":
        # the frames resident on the device: the ring copies device to device
        dev = [{k: api.DeviceArray.from_numpy(ctx, np.ascontiguousarray(f[k]).view(np.uint8))
                for k in ("u", "v", "w", "surface")} for f in src.frames]

    def prefetch(tf):
        if tf not in prefetched:
            k = ((tf - scn.start) // fs) % scn.met.n_frames
            if dev is None:
                f = src.frames[k]
                drv.prefetch_frame(tf, f["u"], f["v"], f["w"], f["surface"])
            else:
                drv.prefetch_frame(tf, *(dev[k][c].ptr for c in ("u", "v", "w", "surface")))
            prefetched.add(tf)

    while drv.has_remaining_steps:
        t = drv.current_time_seconds
        _, _, ta, tb = synthetic.bracket_frames(scn, t)
        if mode in ("ring", "device") and t == scn.start:
            prefetch(ta)
            prefetch(tb)
        if mode == "mixed" and ((ta - scn.start) // fs) % 2 == 0:
            prefetch(ta)
            prefetch(tb)
        drv.run_timestep(src.at(t), forcing)
        if mode in ("ring", "device"):
            prefetch(tb + fs)      # the next bracket's new frame, once this bracket is in use
    drv.finalize()
    return drv.particles.download(), drv.met_ring_stats()


def test_met_ring_streaming_gives_identical_results(ctx):
    scn = _small(particles=20_000, hours=24)
    frames = synthetic.make_frames(scn.met)
    host, (h0, u0) = _run_with_ring(ctx, scn, frames, "host")
    ring, (h1, u1) = _run_with_ring(ctx, scn, frames, "ring")
    mixed, (h2, u2) = _run_with_ring(ctx, scn, frames, "mixed")
    device, (h3, u3) = _run_with_ring(ctx, scn, frames, "device")
    brackets = 8          # 24 h of 3 h brackets
    assert (h0, u0) == (0, brackets)
    assert (h1, u1) == (brackets, 0)
    assert (h2, u2) == (brackets // 2, brackets // 2)
    assert (h3, u3) == (brackets, 0)
    assert host.tobytes() == ring.tobytes() == mixed.tobytes() == device.tobytes()


def test_device_grid_written_as_netcdf_snapshot(ctx, tmp_path):
    from flexpart_gpu import output

    scn = _small(particles=20_000, hours=2)
    frames = synthetic.make_frames(scn.met)
    drv = _driver(ctx, scn)
    src = tl.BracketSource(scn, frames)
    while drv.has_remaining_steps:
        drv.run_timestep(src.at(drv.current_time_seconds), tl.uniform_forcing(dry_velocity=0.002))
    grid = api.Grid(ctx, *scn.out_shape)
    counts, mass, kg = drv.accumulate_concentration_grid(grid, 0, 1e6, scn.outheights)
    path = tmp_path / "grid.nc"
    output.write_grid_netcdf(path, grid, scn.end)
    v = output.read_netcdf(path)["variables"]
    assert v["concentration_particle_count"]["data"].dtype == np.uint32
    assert np.array_equal(v["concentration_particle_count"]["data"].reshape(-1), counts)
    assert np.array_equal(v["concentration_mass_kg"]["data"].reshape(-1), kg)
    assert v["time"]["data"].tolist() == [scn.end]
    assert counts.sum() == 20_000


_SECTIONS = ("sort_ms", "release_ms", "met_bracket_ms", "pbl_ms", "step_ms", "compaction_ms")


def test_step_timing_sections_and_identical_results(ctx):
    """Per-section timing (StepTimingReport, timeloop.rs:398-467): the sections
    are non-negative and add up to the device total, the fused step takes
    time, and turning the timing on changes no result."""
    scn = _small(particles=20_000, hours=2)
    frames = synthetic.make_frames(scn.met)
    forcing = tl.uniform_forcing(dry_velocity=0.002)
    finals = []
    for profile in (False, True):
        drv = _driver(ctx, scn, use_compaction=1, sort_interval_steps=3)
        src = tl.BracketSource(scn, frames)
        if profile:
            drv.set_profiling(True)
        with pytest.raises(api._lib.FpgError) as e:
            drv.last_timing()
        assert e.value.status == -11     # NotReady: no step timed yet
        while drv.has_remaining_steps:
            rep = drv.run_timestep(src.at(drv.current_time_seconds), forcing)
            if not profile:
                continue
            t = drv.last_timing()
            secs = [getattr(t, name) for name in _SECTIONS]
            assert t.step_index == rep.step_index
            assert min(secs) >= 0.0 and t.step_ms > 0.0
            assert abs(sum(secs) - t.gpu_total_ms) <= 0.01 + 1e-3 * t.gpu_total_ms
            assert t.wall_ms >= t.host_call_ms >= 0.0
        finals.append(drv.particles.download())
    assert finals[0].tobytes() == finals[1].tobytes()


def test_profile_environment_variable_prints_one_line_per_step(tmp_path):
    """FLEXPART_GPU_PROFILE=1 at creation prints a [profile] line per step to
    stderr (is_profiling_enabled / print_summary, timeloop.rs:436-476)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = tmp_path / "run.py"
    script.write_text(
        "from flexpart_gpu import api, synthetic, timeloop as tl\n"
        "scn = synthetic.config0()\n"
        "scn.sources[0].particle_count = 2000\nscn.capacity = 2000\nscn.end = scn.start + 3600\n"
        "frames = synthetic.make_frames(scn.met)\n"
        "ctx = api.Context(0)\n"
        "drv = tl.ForwardDriver(ctx, tl.scenario_config(scn), tl.scenario_releases(scn), tl.scenario_domain(scn),\n"
        "                       scn.capacity, (scn.met.nx, scn.met.ny, scn.met.nz))\n"
        "src = tl.BracketSource(scn, frames)\n"
        "n = 0\n"
        "while drv.has_remaining_steps:\n"
        "    drv.run_timestep(src.at(drv.current_time_seconds), tl.uniform_forcing())\n"
        "    n += 1\n"
        "print('steps', n)\n")
    env = dict(os.environ, FLEXPART_GPU_PROFILE="1",
               PYTHONPATH=os.pathsep.join([root, os.path.join(root, "flexpart-gpu_b200")]))
    r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    steps = int(r.stdout.split()[-1])
    lines = [ln for ln in r.stderr.splitlines() if ln.startswith("[profile] step=")]
    assert steps > 0 and len(lines) == steps
    assert all("step=" in ln and "gpu=" in ln and "total=" in ln for ln in lines)


@pytest.mark.parametrize("mode", ["plain", "compaction_sort"])
def test_validation_mode_gives_the_fused_kernels_bits(ctx, mode):
    """The reference's validation path (separated advection, Hanna records,
    Langevin from the records, deposition; timeloop.rs:1128-1155) against the
    fused kernel: identical reports and particle bytes after every step."""
    scn = _small(particles=20_000, hours=4)
    frames = synthetic.make_frames(scn.met)
    kw = {"use_compaction": 1, "sort_interval_steps": 3} if mode == "compaction_sort" else {}
    fused, sep = _driver(ctx, scn, **kw), _driver(ctx, scn, **kw)
    sep.set_validation_mode(True)
    src = tl.BracketSource(scn, frames)
    forcing = tl.uniform_forcing(dry_velocity=0.002, wet_lambda=2e-4, wet_fraction=0.6)
    steps = 0
    while fused.has_remaining_steps:
        ra = fused.run_timestep(src.at(fused.current_time_seconds), forcing)
        rb = sep.run_timestep(src.at(sep.current_time_seconds), forcing)
        assert (ra.released_count, ra.active_particle_count, list(ra.next_philox_counter)) == \
               (rb.released_count, rb.active_particle_count, list(rb.next_philox_counter))
        assert fused.particles.download().tobytes() == sep.particles.download().tobytes(), steps
        steps += 1
    assert steps == 17 and not sep.has_remaining_steps


def test_environment_variables_select_the_separated_path_and_compaction(tmp_path):
    """FLEXPART_GPU_VALIDATION=1 at creation (is_validation_mode,
    timeloop.rs:480-494) runs the separated path, FLEXPART_GPU_COMPACTION=1
    the compaction (as the configuration's use_compaction does)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = tmp_path / "run.py"
    script.write_text(
        "import sys\nimport numpy as np\n"
        "from flexpart_gpu import api, synthetic, timeloop as tl\n"
        "scn = synthetic.config0()\n"
        "scn.sources[0].particle_count = 5000\nscn.capacity = 5000\nscn.end = scn.start + 2 * 3600\n"
        "frames = synthetic.make_frames(scn.met)\n"
        "ctx = api.Context(0)\n"
        "kw = {'use_compaction': 1} if sys.argv[2] == 'cfg_compaction' else {}\n"
        "drv = tl.ForwardDriver(ctx, tl.scenario_config(scn, **kw), tl.scenario_releases(scn),\n"
        "                       tl.scenario_domain(scn), scn.capacity, (scn.met.nx, scn.met.ny, scn.met.nz),\n"
        "                       synthetic.level_heights(scn.met.nz, scn.met.top_m))\n"
        "src = tl.BracketSource(scn, frames)\n"
        "while drv.has_remaining_steps:\n"
        "    drv.run_timestep(src.at(drv.current_time_seconds), tl.uniform_forcing(dry_velocity=0.002))\n"
        "np.save(sys.argv[1], drv.particles.download())\n"
        "print('launches', ctx.kernel_launches)\n")
    runs, launches = {}, {}
    for label, flags in (("separated", {"FLEXPART_GPU_VALIDATION": "1"}), ("fused", {}),
                         ("compaction_env", {"FLEXPART_GPU_COMPACTION": "1"}), ("cfg_compaction", {})):
        env = dict(os.environ, PYTHONPATH=os.pathsep.join([root, os.path.join(root, "flexpart-gpu_b200")]))
        env.pop("FLEXPART_GPU_VALIDATION", None)
        env.pop("FLEXPART_GPU_COMPACTION", None)
        env.update(flags)
        path = tmp_path / f"{label}.npy"
        r = subprocess.run([sys.executable, str(script), str(path), label], env=env, capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        runs[label] = np.load(path)
        launches[label] = int(r.stdout.split()[-1])
    assert runs["separated"].tobytes() == runs["fused"].tobytes()
    assert launches["separated"] > launches["fused"]       # three more passes per step
    # FLEXPART_GPU_COMPACTION=1 (is_compaction_enabled, timeloop.rs:496-513) is
    # the configuration's use_compaction: the same compacted run (its Philox
    # counter advances by the active count, not the capacity)
    assert runs["compaction_env"].tobytes() == runs["cfg_compaction"].tobytes()
    assert launches["compaction_env"] == launches["cfg_compaction"] > launches["fused"]
    assert (runs["fused"]["flags"] & 1).sum() == 5000


def test_run_to_end_with_one_bracket_equals_the_manual_loop(ctx):
    """run_to_end (timeloop.rs:1318-1333): one met bracket and forcing for
    every remaining step (times past the bracket clamped), then finalize; the
    same reports and particles as stepping by hand."""
    scn = _small(particles=10_000, hours=2)
    frames = synthetic.make_frames(scn.met)
    src = tl.BracketSource(scn, frames)
    met = src.at(scn.start)
    forcing = tl.uniform_forcing(dry_velocity=0.002)
    a, b = _driver(ctx, scn, clamp_time_bounds=1), _driver(ctx, scn, clamp_time_bounds=1)
    reports = a.run_to_end(met, forcing)
    manual = []
    while b.has_remaining_steps:
        manual.append(b.run_timestep(met, forcing))
    b.finalize()
    assert len(reports) == len(manual) == 9 and not a.has_remaining_steps
    for ra, rb in zip(reports, manual):
        assert (ra.step_index, ra.released_count, ra.interpolation_alpha, list(ra.next_philox_counter)) == \
               (rb.step_index, rb.released_count, rb.interpolation_alpha, list(rb.next_philox_counter))
    assert a.particles.download().tobytes() == b.particles.download().tobytes()
