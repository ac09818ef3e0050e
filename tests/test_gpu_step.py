"""GPU parity of the fused step and its seam functions against the oracle.

Every call goes through the C ABI (libfpg.so via ctypes).  Tolerance: the
floating-point fields agree to relative 1e-5 of each field's scale after one
step (tests/helpers.py: field_checks); integer fields (cells, flags, cbt) and
Philox outputs are bit-exact.  Against the FP64 oracle the GPU's error is no
larger than the FP32 oracle's own (both printed).
"""
import numpy as np
import pytest

from helpers import (assert_parity, close, fp64_errors, oracle_step, pbl_arrays, population, production_params,
                     small_met)
from oracle import orc

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _gpu_setup(ctx, spec, frames, met, alpha, rec):
    m = api.Met(ctx, spec.nx, spec.ny, spec.nz)
    m.upload_frame(0, met["u0"], met["v0"], met["w0"])
    m.upload_frame(1, met["u1"], met["v1"], met["w1"])
    m.set_level_heights(met["heights"])
    surf = api.Surface(ctx, spec.nx, spec.ny)
    surf.upload(0, frames[0]["surface"])
    surf.upload(1, frames[1]["surface"])
    pbl = api.Pbl(ctx, spec.nx, spec.ny)
    api.pbl_diagnostics(ctx, surf, alpha, pbl)
    p = api.Particles(ctx, len(rec))
    p.upload(rec)
    return m, surf, pbl, p


def _compare_state(g, s, label, rec_in, s64=None):
    stats = assert_parity(g, s, rec_in["pos_z"], s64, label)
    if any(stats.values()):
        print(f"{label}: particles held to the FP32 envelope: {stats}")


def test_philox_kernel_bit_exact(ctx):
    u, raw = api.philox_uniforms(ctx, [0, 0], [0, 0, 0, 0], 1)
    assert list(raw[:4]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    key, ctr = [0xDECAFBAD, 0x12345678], [0xFFFFFFF0, 0xFFFFFFFF, 7, 9]
    u, raw = api.philox_uniforms(ctx, key, ctr, 5000)
    ou, oraw = orc.philox_uniforms(key, ctr, 5000)
    assert np.array_equal(raw, oraw)
    assert np.array_equal(u, ou)


@pytest.mark.parametrize("alpha", [0.0, 0.37, 1.0])
def test_pbl_diagnostics_matches_oracle(ctx, alpha):
    spec, frames, _ = small_met()
    # exercise the fallbacks: missing u*, 1/L, h in some cells
    s0 = frames[0]["surface"].copy()
    s1 = frames[1]["surface"].copy()
    s0["friction_velocity_ms"][::5] = 0.0
    s1["friction_velocity_ms"][::5] = np.nan
    s0["inv_obukhov_length_per_m"][::3] = 0.0
    s1["inv_obukhov_length_per_m"][::3] = 0.0
    s0["mixing_height_m"][::4] = -1.0
    s1["mixing_height_m"][::4] = -1.0
    s0["surface_stress_n_m2"][::7] = 0.0
    s1["surface_stress_n_m2"][::7] = 0.0
    surf = api.Surface(ctx, spec.nx, spec.ny)
    surf.upload(0, s0)
    surf.upload(1, s1)
    pbl = api.Pbl(ctx, spec.nx, spec.ny)
    api.pbl_diagnostics(ctx, surf, alpha, pbl)
    g = pbl.download()
    o = orc.pbl_diagnostics(s0, s1, alpha, spec.nx, spec.ny)
    for k in ("ustar", "wstar", "hmix", "oli", "sshf", "ssr", "surfstr"):
        ok = close(g[k], getattr(o, k), rel=1e-6)
        assert ok.all(), (k, np.flatnonzero(~ok)[:5])


@pytest.mark.parametrize("n", [1, 255, 4099])
def test_fused_step_one_step_matches_oracle(ctx, n):
    spec, frames, met = small_met()
    alpha = 0.3
    rec = population(spec.nx, spec.ny, n)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, alpha, rec)
    prm = production_params(alpha=alpha, counter=(7, 0, 0, 0))
    nxt = api.step(ctx, p, m, pbl, prm)
    g = p.download()
    opbl = pbl_arrays(frames, alpha, spec.nx, spec.ny)
    s = oracle_step(rec, met, opbl, prm)
    s64 = oracle_step(rec, met, pbl_arrays(frames, alpha, spec.nx, spec.ny, np.float64), prm, np.float64)
    _compare_state(g, s, f"n={n}", rec, s64)
    assert nxt == orc.next_counter([7, 0, 0, 0], n, 4)
    # report the error of both against FP64 for every compared field: the
    # GPU is no further from the FP64 restatement than the FP32 oracle is
    act = rec["flags"] == 1
    if not act.any():
        return
    for name, (e_gpu, e_orc) in fp64_errors(g, s, s64, rec["pos_z"], act).items():
        print(f"n={n}: max scaled |{name} - fp64|: gpu {e_gpu:.2e}, oracle f32 {e_orc:.2e}")
        assert e_gpu <= 2.0 * e_orc + 1e-6, name


@pytest.mark.parametrize("n_sub", [0, 1, 2, 3, 4])
def test_substep_counts_and_counter_advance(ctx, n_sub):
    spec, frames, met = small_met(seed=9)
    rec = population(spec.nx, spec.ny, 700, seed=n_sub)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.5, rec)
    prm = production_params(alpha=0.5, n_substeps=n_sub, counter=(0xFFFFFFFE, 0xFFFFFFFF, 3, 0))
    nxt = api.step(ctx, p, m, pbl, prm)
    s = oracle_step(rec, met, pbl_arrays(frames, 0.5, spec.nx, spec.ny), prm)
    s64 = oracle_step(rec, met, pbl_arrays(frames, 0.5, spec.nx, spec.ny, np.float64), prm, np.float64)
    _compare_state(p.download(), s, f"n_sub={n_sub}", rec, s64)
    assert nxt == orc.next_counter([0xFFFFFFFE, 0xFFFFFFFF, 3, 0], 700, n_sub)


def test_legacy_level_index_mode_and_nonmonotonic_heights(ctx):
    for heights in ("legacy", "nonmono"):
        spec, frames, met = small_met(nz=8, heights=heights != "legacy")
        if heights == "nonmono":
            h = met["heights"].copy()
            h[3], h[4] = h[4], h[3]
            met["heights"] = h
        rec = population(spec.nx, spec.ny, 513, z_max=7.0 if heights == "legacy" else 3000.0)
        m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.8, rec)
        prm = production_params(alpha=0.8, stages=1)     # advection only
        api.step(ctx, p, m, pbl, prm)
        s = oracle_step(rec, met, None, prm)
        s64 = oracle_step(rec, met, None, prm, np.float64)
        _compare_state(p.download(), s, heights, rec, s64)


@pytest.mark.parametrize("kind", ["stretched60", "duplicates", "two_levels"])
def test_level_table_search_matches_the_scan(ctx, kind):
    """The bucket-table level search (sorted heights) against the oracle's
    linear scan (advection_dual_wind.wgsl:94-117): heights stretched to
    15 km over 60 levels (several levels per bucket near the ground), heights
    with repeated values, and two levels; particles exactly on level heights,
    one ulp either side of them and of the bucket edges, and at random."""
    if kind == "stretched60":
        nz, hts = 60, (15000.0 * (np.arange(1, 61) / 60.0) ** 2).astype(np.float32)
    elif kind == "duplicates":
        hts = np.array([10, 10, 25, 25, 25, 60, 200, 200, 1000, 5000, 5000, 9000], np.float32)
        nz = len(hts)
    else:
        nz, hts = 2, np.array([50.0, 3000.0], np.float32)
    spec, frames, met = small_met(nz=nz)
    met["heights"] = hts
    rng = np.random.default_rng(nz)
    edges = (hts[0] + (np.arange(1024) * (np.float64(hts[-1]) - hts[0]) / 1024.0)).astype(np.float32)[::7]
    z = np.concatenate([hts, np.nextafter(hts, np.float32(np.inf)), np.nextafter(hts, np.float32(-np.inf)),
                        edges, np.nextafter(edges, np.float32(0)),
                        rng.uniform(0.0, 1.1 * float(hts[-1]), 2000).astype(np.float32)])
    rec = population(spec.nx, spec.ny, len(z), seed=nz, inactive_every=0)
    rec["pos_z"] = z
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.4, rec)
    prm = production_params(alpha=0.4, stages=1)           # advection only
    api.step(ctx, p, m, pbl, prm)
    s = oracle_step(rec, met, None, prm)
    s64 = oracle_step(rec, met, None, prm, np.float64)
    _compare_state(p.download(), s, kind, rec, s64)


def test_bracket_upload_in_one_pass_matches_two_frame_uploads(ctx):
    """fpg_met_upload_bracket_device (both frames, whole nodes) gives the
    bracket of two fpg_met_upload_frame calls: the same step, bit for bit,
    also after a bracket uploaded the other way round first."""
    spec, frames, met = small_met()
    rec = population(spec.nx, spec.ny, 30_001, seed=5)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.3, rec)
    prm = production_params(alpha=0.3, counter=(4, 0, 0, 0))
    api.step(ctx, p, m, pbl, prm)
    want = p.download()
    dev = [api.DeviceArray.from_numpy(ctx, np.ascontiguousarray(met[k], np.float32).reshape(-1))
           for k in ("u0", "v0", "w0", "u1", "v1", "w1")]
    m.upload_bracket_device(dev[3:], dev[:3])          # swapped frames first: every node rewritten
    m.upload_bracket_device(dev[:3], dev[3:])
    p.upload(rec)
    api.step(ctx, p, m, pbl, prm)
    assert p.download().tobytes() == want.tobytes()


def test_launch_shapes_give_the_same_bits_and_the_tuner_restores_the_state(ctx):
    """Every compiled launch shape of fpg_step (block size, resident blocks,
    particles per thread) gives the default shape's results bit for bit;
    fpg_step_autotune leaves the particle state as it found it, keeps a
    compiled shape, and the next step under it matches the default."""
    spec, frames, met = small_met()
    rec = population(spec.nx, spec.ny, 40_001, seed=3)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.6, rec)
    prm = production_params(alpha=0.6, counter=(9, 0, 0, 0))
    shapes = api.step_tuning_candidates()
    out = []
    for t in shapes:
        api.set_step_tuning(ctx, t)
        p.upload(rec)
        api.step(ctx, p, m, pbl, prm)
        out.append(p.download().tobytes())
    assert all(o == out[0] for o in out[1:])
    p.upload(rec)
    best, cands = api.step_autotune(ctx, p, m, pbl, prm, reps=2)
    assert p.download().tobytes() == rec.tobytes()             # state restored
    key = (best["block_threads"], best["min_blocks_per_sm"], best["particles_per_thread"])
    assert key in {(t["block_threads"], t["min_blocks_per_sm"], t["particles_per_thread"]) for t in shapes}
    assert all(c["step_ms"] > 0.0 for c in cands) and best["step_ms"] == min(c["step_ms"] for c in cands)
    got = api.get_step_tuning(ctx)
    assert (got["block_threads"], got["min_blocks_per_sm"], got["particles_per_thread"]) == key
    nxt = api.step(ctx, p, m, pbl, prm)
    assert p.download().tobytes() == out[0]
    assert nxt == orc.next_counter([9, 0, 0, 0], len(rec), 4)
    api.set_step_tuning(ctx, shapes[0])


def test_seam_functions_one_at_a_time(ctx):
    spec, frames, met = small_met(seed=4)
    rec = population(spec.nx, spec.ny, 1000, seed=21, z_max=60.0)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.25, rec)
    opbl = pbl_arrays(frames, 0.25, spec.nx, spec.ny)
    opbl64 = pbl_arrays(frames, 0.25, spec.nx, spec.ny, np.float64)
    s = orc.State.from_records(rec)
    s64 = orc.State.from_records(rec, np.float64)
    # advection (gpu/advection.rs:605)
    api.advect_dual_wind(ctx, p, m, 0.25, 600.0, 2e-5, 3e-5, 1.0)
    prm = production_params(alpha=0.25, dt_seconds=600.0, x_grid_per_meter=2e-5, y_grid_per_meter=3e-5,
                            stages=1)
    orc.step(s, 1000, met, None, prm)
    orc.step(s64, 1000, met, None, prm)
    _compare_state(p.download(), s, "advect", rec, s64)
    # fused Hanna + Langevin (gpu/langevin_fused.rs:133)
    nxt = api.langevin_fused(ctx, p, pbl, 600.0, 2.5e-4, 4, 0.01, (1, 2), (5, 0, 0, 0))
    prm = production_params(stages=2, turb_dt_seconds=600.0, rho_grad_over_rho=2.5e-4, key=(1, 2),
                            counter=(5, 0, 0, 0))
    orc.step(s, 1000, met, opbl, prm)
    orc.step(s64, 1000, met, opbl64, prm)
    _compare_state(p.download(), s, "langevin", rec, s64)
    assert nxt == orc.next_counter([5, 0, 0, 0], 1000, 4)
    # dry deposition with per-slot velocities and probability output (gpu/deposition.rs:315)
    vd = np.linspace(-0.001, 0.05, 1000).astype(np.float32)
    dvd = api.DeviceArray.from_numpy(ctx, vd)
    dprob = api.DeviceArray(ctx, 1000)
    api.dry_deposition(ctx, p, dvd, 600.0, 15.0, dprob)
    oprob = np.zeros(1000, np.float32)
    prm = production_params(stages=4, turb_dt_seconds=600.0, dry_mode=2)
    orc.step(s, 1000, met, None, prm, dry_velocity=vd, dry_prob=oprob)
    orc.step(s64, 1000, met, None, prm, dry_velocity=vd)
    _compare_state(p.download(), s, "dry", rec, s64)
    assert close(dprob.numpy(), oprob).all()
    # wet deposition (gpu/wet_deposition.rs:368)
    lam = np.linspace(0, 3e-3, 1000).astype(np.float32)
    fr = np.linspace(-0.2, 1.3, 1000).astype(np.float32)
    dl, df, wprob = api.DeviceArray.from_numpy(ctx, lam), api.DeviceArray.from_numpy(ctx, fr), api.DeviceArray(ctx, 1000)
    api.wet_deposition(ctx, p, dl, df, 600.0, wprob)
    owprob = np.zeros(1000, np.float32)
    prm = production_params(stages=8, turb_dt_seconds=600.0, dry_mode=0, wet_mode=2)
    orc.step(s, 1000, met, None, prm, wet_lambda=lam, wet_fraction=fr, wet_prob=owprob)
    orc.step(s64, 1000, met, None, prm, wet_lambda=lam, wet_fraction=fr)
    _compare_state(p.download(), s, "wet", rec, s64)
    assert close(wprob.numpy(), owprob).all()


def test_per_cell_wet_forcing_from_precipitation(ctx):
    spec, frames, met = small_met(seed=6)
    rec = population(spec.nx, spec.ny, 3000, seed=8)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.1, rec)
    rng = np.random.default_rng(2)
    lsp = np.where(rng.random(spec.nx * spec.ny) < 0.3, rng.lognormal(-1, 1, spec.nx * spec.ny), 0).astype(np.float32)
    conv = np.where(rng.random(spec.nx * spec.ny) < 0.1, rng.uniform(0, 30, spec.nx * spec.ny), 0).astype(np.float32)
    cc = rng.uniform(0, 1, spec.nx * spec.ny).astype(np.float32)
    cf = api.CellField(ctx, spec.nx, spec.ny)
    cf.from_precipitation(lsp, conv, cc, 1e-4, 0.8)
    lam, fr = orc.wet_cells(lsp, conv, cc, 1e-4, 0.8)
    prm = production_params(alpha=0.1, wet_mode=3)
    api.step(ctx, p, m, pbl, prm, wet_cells=cf)
    kw = dict(wet_cells_lf=(lam, fr), wet_shape=(spec.nx, spec.ny))
    s = oracle_step(rec, met, pbl_arrays(frames, 0.1, spec.nx, spec.ny), prm, **kw)
    s64 = oracle_step(rec, met, pbl_arrays(frames, 0.1, spec.nx, spec.ny, np.float64), prm, np.float64, **kw)
    _compare_state(p.download(), s, "per-cell wet", rec, s64)


def test_empty_and_all_inactive(ctx):
    spec, frames, met = small_met()
    rec = population(spec.nx, spec.ny, 300)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.0, rec)
    p.dispatch_count = 0
    prm = production_params(counter=(9, 0, 0, 0))
    assert api.step(ctx, p, m, pbl, prm) == [9, 0, 0, 0]       # empty: Ok, counter unchanged
    assert np.array_equal(p.download(), rec)
    rec2 = rec.copy()
    rec2["flags"] = 0
    p.dispatch_count = 300
    p.upload(rec2)
    api.step(ctx, p, m, pbl, prm)
    assert np.array_equal(p.download(), rec2)


def test_error_codes_mirror_reference(ctx):
    spec, frames, met = small_met()
    rec = population(spec.nx, spec.ny, 10)
    m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.0, rec)
    with pytest.raises(api._lib.FpgError) as e:
        api.step(ctx, p, m, pbl, production_params(turb_dt_seconds=0.0))
    assert e.value.status == -2          # InvalidTimeStep (langevin_fused.rs:147)
    with pytest.raises(api._lib.FpgError) as e:
        api.step(ctx, p, m, pbl, production_params(dt_seconds=float("nan"), stages=1))
    assert e.value.status == -2          # gpu/advection.rs:618
    with pytest.raises(api._lib.FpgError) as e:
        api.step(ctx, p, m, pbl, production_params(dry_reference_height_m=0.0, stages=4))
    assert e.value.status == -8          # InvalidReferenceHeight
    with pytest.raises(api._lib.FpgError) as e:
        api.Met(ctx, 0, 4, 4)
    assert e.value.status == -3          # ZeroShape
    m2 = api.Met(ctx, 4, 4, 4)
    with pytest.raises(api._lib.FpgError) as e:
        api.step(ctx, p, m2, pbl, production_params(stages=1))
    assert e.value.status == -11         # bracket never uploaded
    g = api.Grid(ctx, 4, 4, 2)
    with pytest.raises(api._lib.FpgError) as e:
        g.accumulate(p, species=4)
    assert e.value.status == -6          # InvalidSpeciesIndex
    with pytest.raises(api._lib.FpgError) as e:
        g.accumulate(p, mass_scale=0.0)
    assert e.value.status == -7          # InvalidMassScale
    # the failed calls left the particles untouched
    assert np.array_equal(p.download(), rec)


def test_surface_and_precipitation_accept_device_arrays(ctx):
    """A caller whose met is already in HBM passes device pointers for the
    surface frames and the precipitation: the PBL, and a step with the
    per-cell wet forcing, come out bit for bit as from host arrays."""
    import ctypes

    spec, frames, met = small_met(seed=3)
    lib = api._lib.lib
    n = spec.nx * spec.ny
    rng = np.random.default_rng(4)
    lsp = np.where(rng.random(n) < 0.3, rng.lognormal(-1, 1, n), 0).astype(np.float32)
    rec = population(spec.nx, spec.ny, 3000, seed=12)
    out = {}
    for label in ("host", "device"):
        m, surf, pbl, p = _gpu_setup(ctx, spec, frames, met, 0.3, rec)
        cf = api.CellField(ctx, spec.nx, spec.ny)
        if label == "host":
            cf.from_precipitation(lsp, None, None, 1e-4, 0.8)
        else:
            keep = [api.DeviceArray.from_numpy(ctx, frames[k]["surface"].view(np.uint8)) for k in (0, 1)]
            d_lsp = api.DeviceArray.from_numpy(ctx, lsp)
            for k in (0, 1):
                surf.upload(k, np.zeros_like(frames[k]["surface"]))       # overwritten by the device copy
                api.check(lib.fpg_surface_upload(surf.h, k, ctypes.c_void_p(keep[k].ptr), None), "surface")
            api.check(lib.fpg_cellfield_from_precipitation(cf.h, ctypes.c_void_p(d_lsp.ptr), None, None, 1e-4, 0.8,
                                                           None), "wet cells")
            api.pbl_diagnostics(ctx, surf, 0.3, pbl)
        api.step(ctx, p, m, pbl, production_params(alpha=0.3, wet_mode=3), wet_cells=cf)
        out[label] = (pbl.download(), p.download().tobytes())
    for k in ("ustar", "wstar", "hmix", "oli", "sshf", "ssr", "surfstr"):
        assert out["host"][0][k].tobytes() == out["device"][0][k].tobytes(), k
    assert out["host"][1] == out["device"][1]
