"""The batched ensemble (fpg_batch_*): scenarios with uneven particle counts,
their own sources, start times and Philox keys, stepped as one population.

* The graph-replayed batched step, the same kernels launched one by one and
  the sequential path (one plain fused-step launch per scenario per step)
  give bit-identical particles and per-scenario grids.
* Each scenario's particles and grid are bit-identical to a plain forward
  driver run of that release alone (capacity = its particle count, its key).
"""
import numpy as np
import pytest

from flexpart_gpu import synthetic
from flexpart_gpu._lib import FpgError

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")
tl = pytest.importorskip("flexpart_gpu.timeloop")
bt = pytest.importorskip("flexpart_gpu.batch")


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _ensemble(n=9, hours=6):
    met = synthetic.MetSpec(nx=40, ny=30, nz=16, dx_deg=1.0, dy_deg=1.0, xlon0=-20.0, ylat0=30.0, n_frames=3,
                            frame_seconds=3600, seed=5, wet=True)
    ens = synthetic.config2(n_scenarios=n, lo=200, hi=30_000, hours=hours, met=met, seed=11)
    # edge cases: a scenario below one tile, one of exactly one tile, a point release (start == end)
    ens.sources[0].particle_count = 97
    ens.sources[1].particle_count = 256
    ens.sources[2].end = ens.sources[2].start
    return ens


def _batch(ctx, ens, every):
    b = bt.Batch(ctx, bt.ensemble_config(ens, output_every_steps=every), bt.ensemble_scenarios(ens),
                 (ens.met.nx, ens.met.ny, ens.met.nz), synthetic.level_heights(ens.met.nz, ens.met.top_m),
                 ens.outheights)
    frames, precs = bt.upload_ensemble_met(b, ens)
    return b, frames, precs


def test_graph_eager_and_sequential_paths_are_bit_identical(ctx):
    ens = _ensemble()
    every = 5
    n = ens.n_steps  # 25 steps: the last is an output step
    outs = []
    for mode in ("graph", "eager", "sequential"):
        b, _, _ = _batch(ctx, ens, every)
        # two calls, so graph replay continues from a state the previous call left
        for chunk in (7, n - 7):
            if mode == "sequential":
                b.run_sequential(chunk)
            else:
                b.run(chunk, graph=(mode == "graph"))
        assert b.steps_done == n
        with pytest.raises(FpgError):
            b.run(1)
        assert b.errors() == 0
        outs.append((b.particles.download(), *b.download_grids()))
        del b
    ref = outs[0]
    for other in outs[1:]:
        assert ref[0].tobytes() == other[0].tobytes()
        assert np.array_equal(ref[1], other[1])
        assert np.array_equal(ref[2], other[2])
    # every released particle was gridded at the last output step
    counts = ref[1].reshape(len(ens.sources), -1).sum(axis=1)
    for s, src in enumerate(ens.sources):
        b_first = sum(((x.particle_count + 255) // 256) * 256 for x in ens.sources[:s])
        seg = ref[0][b_first:b_first + src.particle_count]
        active = int((seg["flags"] & 1).sum())
        assert counts[s] == active


@pytest.mark.parametrize("s", [0, 2, 4, 8])
def test_scenario_matches_a_plain_driver_run_bit_for_bit(ctx, s):
    ens = _ensemble()
    every = 5
    n = ens.n_steps
    b, frames, precs = _batch(ctx, ens, every)
    b.run(n)
    pop = b.particles.download()
    counts, mass = b.download_grids()
    first, count = b.slots(s)
    assert count == ens.sources[s].particle_count
    assert first % 256 == 0

    scn = ens.scenario(s)
    cfg = tl.scenario_config(scn)
    drv = tl.ForwardDriver(ctx, cfg, tl.scenario_releases(scn), tl.scenario_domain(scn), count,
                           (ens.met.nx, ens.met.ny, ens.met.nz), synthetic.level_heights(ens.met.nz, ens.met.top_m))
    src = tl.BracketSource(scn, frames)
    cells = api.CellField(ctx, ens.met.nx, ens.met.ny)
    forcing = tl.cell_forcing(cells, dry_velocity=ens.dry_velocity)
    last_fa = None
    for _ in range(n):
        t = drv.current_time_seconds
        fa, _, _, _ = synthetic.bracket_frames(scn, t)
        if fa != last_fa:
            cells.from_precipitation(precs[fa], a=ens.wet_a, b=ens.wet_b)
            last_fa = fa
        drv.run_timestep(src.at(t), forcing)
    drv.finalize()
    plain = drv.particles.download()
    assert pop[first:first + count].tobytes() == plain.tobytes()
    grid = api.Grid(ctx, *ens.out_shape)
    gc, gm, _ = drv.accumulate_concentration_grid(grid, outheights=ens.outheights)
    assert np.array_equal(counts[s].reshape(-1), gc)
    assert np.array_equal(mass[s].reshape(-1), gm)
    del drv


def test_batch_errors(ctx):
    ens = _ensemble(n=3)
    cfg = bt.ensemble_config(ens)
    scen = bt.ensemble_scenarios(ens)
    shape = (ens.met.nx, ens.met.ny, ens.met.nz)
    # a release outside the release grid
    scen[1].release.lon_min = scen[1].release.lon_max = ens.met.xlon0 - 5.0
    with pytest.raises(FpgError) as e:
        bt.Batch(ctx, cfg, scen, shape)
    assert e.value.status == -16
    scen = bt.ensemble_scenarios(ens)
    scen[0].release.particle_count = 0
    with pytest.raises(FpgError):
        bt.Batch(ctx, cfg, scen, shape)
    scen = bt.ensemble_scenarios(ens)
    scen[0].release.lat_min, scen[0].release.lat_max = 5.0, 1.0
    with pytest.raises(FpgError) as e:
        bt.Batch(ctx, cfg, scen, shape)
    assert e.value.status == -15
    cfg.end_seconds = cfg.start_seconds - 1
    with pytest.raises(FpgError) as e:
        bt.Batch(ctx, cfg, bt.ensemble_scenarios(ens), shape)
    assert e.value.status == -18


def test_every_launch_shape_and_the_tuner_leave_results_unchanged(ctx):
    ens = _ensemble()
    n = ens.n_steps
    b, _, _ = _batch(ctx, ens, 5)
    b.run(n)
    ref = (b.particles.download().tobytes(), *b.download_grids())
    del b
    for t in bt.tuning_candidates():
        b, _, _ = _batch(ctx, ens, 5)
        b.tuning = t
        assert b.tuning["block_threads"] == t["block_threads"]
        b.run(n)
        got = (b.particles.download().tobytes(), *b.download_grids())
        assert got[0] == ref[0], t
        assert np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2]), t
        del b
    # tuning in the middle of a run: the trial steps are undone
    b, _, _ = _batch(ctx, ens, 5)
    b.run(12)
    best, allc = b.autotune(reps=2)
    assert len(allc) == len(bt.tuning_candidates())
    assert all(c["step_ms"] > 0.0 for c in allc)
    assert best["step_ms"] == min(c["step_ms"] for c in allc)
    assert b.tuning["block_threads"] == best["block_threads"]
    assert b.steps_done == 12
    b.run(n - 12)
    got = (b.particles.download().tobytes(), *b.download_grids())
    assert got[0] == ref[0]
    assert np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])
    with pytest.raises(FpgError):
        b.tuning = {"block_threads": 96, "min_blocks_per_sm": 1, "particles_per_thread": 1}
