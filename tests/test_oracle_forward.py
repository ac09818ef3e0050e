"""The oracle's forward loop reproduces the reference's time-loop tests:
alpha sequence, release counts per step, inclusive step count, counter
chaining (CPU only)."""
import numpy as np

from flexpart_gpu import synthetic
from oracle import orc
from oracle.forward import OracleForward


def _tiny_scenario():
    scn = synthetic.config0()
    scn.met = synthetic.MetSpec(nx=30, ny=20, nz=10, dx_deg=0.5, dy_deg=0.5, xlon0=-10.0, ylat0=35.0,
                                n_frames=2, seed=0)
    scn.sources[0].lon, scn.sources[0].lat = -10.0 + 5.25, 35.0 + 5.25
    scn.sources[0].particle_count = 2000
    scn.capacity = 2000
    scn.end = scn.start + 4 * 3600
    scn.out_shape = (30, 20, 3)
    return scn


def test_forward_loop_release_alpha_and_counter_chain():
    scn = _tiny_scenario()
    frames = synthetic.make_frames(scn.met)
    fw = OracleForward(scn, 2000, frames)
    reports = []
    while fw.has_remaining_steps:
        reports.append(fw.run_timestep({"dry_velocity": 0.002}))
    # inclusive loop (timeloop.rs:832-834): 4 h / 900 s + 1 steps
    assert len(reports) == 17
    # emission over [start, start+1h]: 0 at the start, then 500 per 15 min (release/mod.rs:181-196)
    assert [r["released"] for r in reports[:6]] == [0, 500, 500, 500, 500, 0]
    assert reports[-1]["active"] == 2000
    # alpha within the 3 h bracket: 0, 1/12, ... , then the next bracket restarts at 1/12
    assert [round(r["alpha"], 6) for r in reports[:3]] == [0.0, round(1 / 12, 6), round(2 / 12, 6)]
    assert reports[12]["alpha"] == 1.0
    # counter advances by capacity * 2 blocks per step (gpu/langevin_fused.rs:229-233)
    assert reports[0]["counter"] == [4000, 0, 0, 0]
    assert reports[-1]["counter"] == [4000 * 17, 0, 0, 0]
    # the mass budget: nothing leaves, dry deposition only decays mass
    g_counts, g_mass, _ = fw.grid()
    assert g_counts.sum() == 2000


def test_forward_loop_alpha_sequence_of_reference_test():
    # tests/forward_timeloop.rs:100-126: bracket [t0, t0+2], dt 1 -> alpha 0, 0.5, 1
    for k, a in enumerate([0.0, 0.5, 1.0]):
        assert orc.interpolation_alpha(10, 12, 10 + k) == (0, a)


def test_sampled_step_with_slot_indices_equals_population_step():
    """orc.step on a sample of slots, each keeping its Philox index through
    rng_index, gives the same bits as the step of the whole population at
    those slots (the sampled parity tests at full size rely on it)."""
    from helpers import oracle_step, pbl_arrays, population, production_params, small_met

    spec, frames, met = small_met()
    rec = population(spec.nx, spec.ny, 3000, seed=4)
    prm = production_params(alpha=0.6, counter=(11, 0, 0, 0))
    pbl = pbl_arrays(frames, 0.6, spec.nx, spec.ny)
    full = oracle_step(rec, met, pbl, prm).to_records()
    slots = np.sort(np.random.default_rng(1).choice(3000, 400, replace=False)).astype(np.uint32)
    st = orc.State.from_records(rec[slots])
    orc.step(st, len(slots), met, pbl, prm, rng_index=slots)
    assert st.to_records().tobytes() == full[slots].tobytes()
    # without the indices the sample draws other noise
    st2 = orc.State.from_records(rec[slots])
    orc.step(st2, len(slots), met, pbl, prm)
    assert st2.to_records().tobytes() != full[slots].tobytes()
