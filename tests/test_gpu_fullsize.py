"""Full-size checks through size-independent properties (the oracle is too
slow for a whole 10 M-particle population or the 54 M-particle ensemble):

* 10 M particles of the global run (configuration 1 sizes): with deposition
  off every particle's mass is unchanged bit for bit; with it on every mass
  is scaled by a survival factor in (0, 1]; the step is deterministic;
* the reorder by met cell leaves the cell keys non-decreasing (keys
  recomputed by the oracle from the device's own positions) and permutes
  the population (same multiset of records);
* the grid's counts sum to the active particles and its masses to the sum
  of their quantised masses (bit-exact integer arithmetic);
* compaction with 30 % of slots inactive keeps the active records in slot
  order and is idempotent;
* the batched 256-scenario ensemble (54 M particles, 97 steps): graph replay
  and one plain launch per scenario per step give the same bits.
"""
import numpy as np
import pytest

from flexpart_gpu import synthetic
from flexpart_gpu.records import StepParams

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")

N = 10_000_000


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def world(ctx):
    scn = synthetic.config1(N)
    spec = scn.met
    frames = synthetic.make_frames(spec)
    met = api.Met(ctx, spec.nx, spec.ny, spec.nz)
    met.set_level_heights(synthetic.level_heights(spec.nz, spec.top_m))
    met.upload_frame(0, frames[0]["u"], frames[0]["v"], frames[0]["w"])
    met.upload_frame(1, frames[1]["u"], frames[1]["v"], frames[1]["w"])
    surf = api.Surface(ctx, spec.nx, spec.ny)
    surf.upload(0, frames[0]["surface"])
    surf.upload(1, frames[1]["surface"])
    pbl = api.Pbl(ctx, spec.nx, spec.ny)
    api.pbl_diagnostics(ctx, surf, 0.4, pbl)
    rec = synthetic.particles_at_sources(scn, N, seed=21)
    return scn, met, pbl, rec


def _params(scn, **kw):
    xs, ys, zs = synthetic.velocity_scale(scn.met)
    return StepParams.production(alpha=0.4, dt_seconds=900.0, turb_dt_seconds=900.0, x_grid_per_meter=xs,
                                 y_grid_per_meter=ys, z_grid_per_meter=zs, key=(7, 9), counter=(3, 0, 0, 0), **kw)


def test_full_size_step_mass_conservation_and_determinism(ctx, world):
    scn, met, pbl, rec = world
    parts = api.Particles(ctx, N)
    parts.upload(rec)
    api.step(ctx, parts, met, pbl, _params(scn))
    a = parts.download()
    assert np.array_equal(a["mass"], rec["mass"])               # no deposition: masses untouched
    moved = (a["pos_x"] != rec["pos_x"]) | (a["cell_x"] != rec["cell_x"])
    assert moved.mean() > 0.99
    parts.upload(rec)
    api.step(ctx, parts, met, pbl, _params(scn))
    assert parts.download().tobytes() == a.tobytes()           # deterministic
    parts.upload(rec)
    api.step(ctx, parts, met, pbl, _params(scn, dry_mode=1, dry_velocity_m_s=0.01))
    d = parts.download()
    ratio = d["mass"][:, 0].astype(np.float64) / rec["mass"][:, 0].astype(np.float64)
    assert np.all(ratio <= 1.0) and np.all(ratio > 0.0)
    assert (ratio < 1.0).any() and (ratio == 1.0).any()      # near-ground particles decay, others do not


def test_full_size_reorder_sorts_and_permutes(ctx, world):
    from oracle import orc

    scn, met, pbl, rec = world
    spec = scn.met
    parts = api.Particles(ctx, N)
    r = rec.copy()
    r["time"] = np.arange(N, dtype=np.int32)                    # a tag that follows each particle
    parts.upload(r)
    api.step(ctx, parts, met, pbl, _params(scn))
    before = parts.download()
    api.Sorter(ctx, N).sort(parts, met)
    after = parts.download()
    keys = orc.cell_keys(orc.State.from_records(after), N, synthetic.level_heights(spec.nz, spec.top_m),
                         (spec.nx, spec.ny, spec.nz))
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    # a permutation: every tag once, each record unchanged
    assert np.array_equal(np.sort(after["time"]), np.arange(N, dtype=np.int32))
    assert after[np.argsort(after["time"])].tobytes() == before.tobytes()


def test_full_size_grid_totals(ctx, world):
    scn, met, pbl, rec = world
    parts = api.Particles(ctx, N)
    r = rec.copy()
    r["flags"][::7] = 0                                         # some inactive slots
    r["mass"][:, 0] = np.random.default_rng(2).uniform(1e-6, 1e-4, N).astype(np.float32)
    parts.upload(r)
    grid = api.Grid(ctx, *scn.out_shape)
    grid.accumulate(parts, 0, 1e6, scn.outheights)
    counts, mass, _ = grid.download()
    act = (r["flags"] & 1) != 0
    assert int(counts.astype(np.int64).sum()) == int(act.sum())
    q = np.floor(r["mass"][act, 0].astype(np.float32) * np.float32(1e6) + np.float32(0.5)).astype(np.int64)
    assert q.sum() < 2**32                                      # so no cell can wrap
    assert int(mass.astype(np.int64).sum()) == int(q.sum())


def test_full_size_compaction_stable_and_idempotent(ctx, world):
    scn, met, pbl, rec = world
    rng = np.random.default_rng(5)
    r = rec.copy()
    r["flags"][rng.random(N) < 0.3] = 0
    r["time"] = np.arange(N, dtype=np.int32)                    # slot tag to check the order
    parts = api.Particles(ctx, N)
    parts.upload(r)
    comp = api.Compaction(ctx, N)
    n1 = comp.compact(parts)
    act = (r["flags"] & 1) != 0
    assert n1 == int(act.sum())
    c1 = parts.download()
    assert np.array_equal(c1["time"][:n1], np.flatnonzero(act).astype(np.int32))
    assert not (c1["flags"][n1:] & 1).any()
    n2 = comp.compact(parts)
    assert n2 == n1
    assert parts.download().tobytes() == c1.tobytes()


def test_full_size_batched_ensemble_graph_equals_sequential(ctx):
    bt = pytest.importorskip("flexpart_gpu.batch")
    ens = synthetic.config2()
    frames = synthetic.make_frames(ens.met)
    precs = [synthetic.precipitation(ens.met, k) for k in range(ens.met.n_frames)]
    out = []
    for mode in ("graph", "sequential"):
        b = bt.Batch(ctx, bt.ensemble_config(ens, output_every_steps=12), bt.ensemble_scenarios(ens),
                     (ens.met.nx, ens.met.ny, ens.met.nz), synthetic.level_heights(ens.met.nz, ens.met.top_m),
                     ens.outheights)
        for k, f in enumerate(frames):
            b.upload_frame(k, f, precs[k])
        if mode == "graph":
            b.run(ens.n_steps)
        else:
            b.run_sequential(ens.n_steps)
        assert b.errors() == 0
        p = b.particles
        fields = tuple(p.read_field(f).tobytes() for f in ("pos_x", "pos_y", "pos_z", "cell_x", "turb_w", "mass0"))
        active = int((p.read_field("flags") & 1).sum())
        c, m = b.download_grids()
        out.append((fields, active, c, m))
        del b, p
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][2], out[1][2]) and np.array_equal(out[0][3], out[1][3])
    assert out[0][1] == out[1][1] and out[0][1] > 0
