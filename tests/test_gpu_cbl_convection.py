"""CBL sampling, per-slot Hanna parameters and convective mixing on the GPU,
against the oracle.

Tolerances are the reference's own GPU-vs-CPU bars: 5e-5 relative (and
absolute) per field, 5e-4 for the third moment and the skewness
(src/gpu/cbl.rs:446-515), 5e-5 for the Hanna records (src/gpu/hanna.rs:405).
Convective mixing is bit-exact: the destination height of a level is the
same sequential f32 sum on both sides.
"""
import numpy as np
import pytest

from oracle import orc

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")

IFACE = [0.0, 400.0, 1000.0, 2000.0, 3500.0, 5000.0]
TOL = {"third_moment_w3": 5e-4, "skewness": 5e-4, "z_over_h": 5e-6}


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _close(a, b, rel, absol):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= np.maximum(absol, rel * np.maximum(np.abs(a), np.abs(b)))


def _records(xyz, active=None):
    from flexpart_gpu.records import PARTICLE_DTYPE
    xyz = np.asarray(xyz, np.float64)
    rec = np.zeros(len(xyz), PARTICLE_DTYPE)
    cx = np.floor(xyz[:, 0]).astype(np.int32)
    cy = np.floor(xyz[:, 1]).astype(np.int32)
    rec["cell_x"], rec["cell_y"] = cx, cy
    rec["pos_x"] = (xyz[:, 0] - cx).astype(np.float32)
    rec["pos_y"] = (xyz[:, 1] - cy).astype(np.float32)
    rec["pos_z"] = xyz[:, 2].astype(np.float32)
    rec["flags"] = 1 if active is None else np.asarray(active, np.uint32)
    rec["mass"][:, 0] = 1.0
    return rec


def _upload(ctx, rec):
    p = api.Particles(ctx, rec.size)
    p.upload(rec)
    return p


def _compare_outputs(gpu, ref, skip_sample=None):
    from flexpart_gpu.records import CBL_OUTPUT_DTYPE
    for k, name in enumerate(CBL_OUTPUT_DTYPE.names):
        tol = TOL.get(name, 5e-5)
        ok = _close(gpu[name], ref[:, k], tol, tol)
        if name == "sampled_w_m_s" and skip_sample is not None:
            ok |= skip_sample
        assert ok.all(), (name, np.flatnonzero(~ok)[:5], gpu[name][~ok][:5], ref[~ok, k][:5])


def test_cbl_sampling_matches_the_reference_test_case(ctx):
    # src/gpu/cbl.rs:522-594: four particles, the last inactive
    from flexpart_gpu import cbl
    rec = _records([(0.2, 0.0, 120.0), (1.2, 0.0, 80.0), (2.0, 0.0, 200.0), (3.0, 0.0, 30.0)], [1, 1, 1, 0])
    hin = [(0.30, 1.80, -50.0, 900.0, 120.0), (0.25, 0.0, float("inf"), 800.0, 80.0),
           (0.35, 0.0, 100.0, 700.0, 200.0), (0.2, 0.0, 80.0, 600.0, 30.0)]
    hanna = np.zeros(4, cbl.HANNA_PARAMS_DTYPE)
    for i, (u, w, ol, h, z) in enumerate(hin):
        d = orc.hanna(u, w, ol, h, z)
        for k, v in d.items():
            hanna[k][i] = v
    inputs = cbl.sampling_inputs([0.1, 0.8, 0.2, 0.4], [0.4, 0.9, 0.6, 0.1], [0.7, 0.3, 0.5, 0.2])
    gpu = cbl.sample_cbl_vertical_velocity_gpu(ctx, _upload(ctx, rec), hanna, inputs)
    ref = orc.cbl_sample_slots(rec, hanna, inputs)
    _compare_outputs(gpu, ref)
    assert np.all(gpu.view(np.float32).reshape(4, 12)[3] == 0.0)      # inactive: zeroed output


def _hanna_records(rec, rng, nx=50, ny=50):
    """HannaParams of the oracle at each slot's cell of a random PBL."""
    from flexpart_gpu.records import HANNA_PARAMS_DTYPE
    ust, hmix, oli = rng.uniform(0.05, 0.8, (nx, ny)), rng.uniform(50, 2500, (nx, ny)), rng.uniform(-0.2, 0.05, (nx, ny))
    h = orc.hanna_params_slots(rec, ust, _wstar(ust, hmix, oli), hmix, oli, nx, ny)
    out = np.zeros(rec.size, HANNA_PARAMS_DTYPE)
    out.view(np.float32).reshape(rec.size, 16)[:] = h
    return out


def test_cbl_sampling_matches_the_oracle_on_random_slots(ctx):
    """Slots over a random PBL, each with its Hanna record: the PDF and the
    sample within the reference's own GPU-vs-CPU tolerance."""
    from flexpart_gpu import cbl
    rng = np.random.default_rng(11)
    n = 200_000
    rec = _records(np.c_[rng.uniform(0, 50, n), rng.uniform(0, 50, n), rng.uniform(-50, 3000, n)],
                   (rng.random(n) > 0.1).astype(np.uint32))
    hanna = _hanna_records(rec, rng)
    inputs = cbl.sampling_inputs(rng.random(n, np.float32), rng.random(n, np.float32), rng.random(n, np.float32))
    gpu = cbl.sample_cbl_vertical_velocity_gpu(ctx, _upload(ctx, rec), hanna, inputs)
    ref = orc.cbl_sample_slots(rec, hanna, inputs)
    # a branch uniform within 1e-5 of the updraft weight may fall on either side
    near = np.abs(inputs["branch_uniform"].astype(np.float64) - ref[:, 1]) < 1e-5
    _compare_outputs(gpu, ref, skip_sample=near)
    assert near.mean() < 1e-3


def test_cbl_pdf_at_extreme_skewness(ctx):
    """sigma_w far below w* (skewness up to ~1e3, outside what Hanna gives):
    the updraft weight 0.5 * (1 - x / sqrt(4 + r)) cancels to a few 1e-3,
    so single-ulp differences of cbrt / pow grow to a few 1e-4 relative in
    the branch means.  The PDF stays a proper mixture and within 1e-3 of
    the oracle."""
    from flexpart_gpu import cbl
    rng = np.random.default_rng(12)
    n = 100_000
    rec = _records(np.c_[np.full(n, 0.5), np.full(n, 0.5), rng.uniform(0, 3000, n)])
    hanna = np.zeros(n, cbl.HANNA_PARAMS_DTYPE)
    hanna["h"] = rng.uniform(50, 2500, n)
    hanna["wst"] = rng.uniform(0, 3.5, n)
    hanna["sigw"] = rng.uniform(0.05, 2.0, n)
    hanna["ol"] = -rng.uniform(5, 500, n)
    inputs = cbl.sampling_inputs(rng.random(n, np.float32), rng.random(n, np.float32), rng.random(n, np.float32))
    gpu = cbl.sample_cbl_vertical_velocity_gpu(ctx, _upload(ctx, rec), hanna, inputs)
    ref = orc.cbl_sample_slots(rec, hanna, inputs)
    w = gpu["updraft_weight"].astype(np.float64) + gpu["downdraft_weight"]
    assert np.all(np.abs(w - 1.0) < 1e-6)
    assert np.all((gpu["updraft_weight"] > 0) & (gpu["updraft_weight"] < 1))
    assert np.all((gpu["updraft_sigma_m_s"] > 0) & (gpu["downdraft_sigma_m_s"] > 0))
    assert np.all(gpu["updraft_mean_m_s"] >= 0) and np.all(gpu["downdraft_mean_m_s"] <= 0)
    for k, name in enumerate(cbl.CBL_OUTPUT_DTYPE.names[1:], start=1):
        assert _close(gpu[name], ref[:, k], 1e-3, 1e-5).all(), name


def _wstar(ust, hmix, oli):
    """w* consistent with u*, h and L, as the PBL diagnostics relate them:
    w*^3 = -u*^3 h / (kappa L) in unstable cells (kappa = 0.4), else 0."""
    return np.where(oli < -1e-5, ust * np.cbrt(np.maximum(-hmix * oli / 0.4, 0.0)), 0.0).astype(np.float32)


def _pbl(ctx, nx, ny, rng):
    ust = rng.uniform(0.05, 0.8, (nx, ny)).astype(np.float32)
    hmix = rng.uniform(100.0, 2500.0, (nx, ny)).astype(np.float32)
    oli = rng.uniform(-0.05, 0.02, (nx, ny)).astype(np.float32)
    oli[rng.random((nx, ny)) < 0.1] = 0.0
    wst = _wstar(ust, hmix, oli)
    pbl = api.Pbl(ctx, nx, ny)
    pbl.upload(ust, wst, hmix, oli)
    return pbl, (ust, wst, hmix, oli)


def test_hanna_params_match_the_oracle(ctx):
    from flexpart_gpu import cbl
    rng = np.random.default_rng(5)
    nx, ny, n = 40, 30, 100_000
    pbl, fields = _pbl(ctx, nx, ny, rng)
    rec = _records(np.c_[rng.uniform(-2, nx + 2, n), rng.uniform(-2, ny + 2, n), rng.uniform(-10, 3000, n)],
                   (rng.random(n) > 0.2).astype(np.uint32))
    gpu = cbl.compute_hanna_params_gpu(ctx, _upload(ctx, rec), pbl)
    ref = orc.hanna_params_slots(rec, *fields, nx, ny)
    g = gpu.view(np.float32).reshape(n, 16)
    for k, name in enumerate(cbl.HANNA_PARAMS_DTYPE.names[:13]):
        fin = np.isfinite(ref[:, k])
        assert np.array_equal(np.isfinite(g[:, k]), fin), name
        ok = _close(g[fin, k], ref[fin, k], 5e-5, 5e-5)
        assert ok.all(), (name, g[fin, k][~ok][:5], ref[fin, k][~ok][:5])
    assert np.all(g[rec["flags"] == 0] == 0.0)


def test_fused_philox_sampler_matches_the_oracle_chain(ctx):
    """fpg_cbl_sample_philox = Hanna at the slot's cell + the uniforms of
    Philox block counter + slot + the sampler, all in the oracle."""
    from flexpart_gpu import cbl
    rng = np.random.default_rng(8)
    nx, ny, n = 20, 20, 100_000
    pbl, fields = _pbl(ctx, nx, ny, rng)
    rec = _records(np.c_[rng.uniform(0, nx, n), rng.uniform(0, ny, n), rng.uniform(0, 2500, n)],
                   (rng.random(n) > 0.1).astype(np.uint32))
    key, counter = [0xCAFEBABE, 0x12345678], [7, 11, 13, 17]
    gpu = cbl.sample_cbl_vertical_velocity_philox(ctx, _upload(ctx, rec), pbl, key, counter)
    hanna = orc.hanna_params_slots(rec, *fields, nx, ny)
    u, _ = orc.philox_uniforms(key, counter, n)
    u = u.reshape(n, 4)
    inputs = cbl.sampling_inputs(u[:, 0], u[:, 1], u[:, 2])
    ref = orc.cbl_sample_slots(rec, hanna, inputs)
    near = np.abs(u[:, 0].astype(np.float64) - ref[:, 1]) < 1e-5
    _compare_outputs(gpu, ref, skip_sample=near)


def test_fused_sampler_reproduces_the_target_moments(ctx):
    """The moment check of physics/cbl.rs:376-420 on the device: one
    convective column, 2 M slots at one height, each with its own Philox
    block; the sample moments match the PDF's target moments."""
    from flexpart_gpu import cbl
    n = 2_000_000
    pbl = api.Pbl(ctx, 1, 1)
    pbl.upload([0.35], [2.4], [1400.0], [-1.0 / 90.0])
    rec = _records(np.tile([0.5, 0.5, 200.0], (n, 1)))
    out = cbl.sample_cbl_vertical_velocity_philox(ctx, _upload(ctx, rec), pbl, [0xCAFEBABE, 0x12345678],
                                                  [7, 11, 13, 17])
    w = out["sampled_w_m_s"].astype(np.float64)
    assert abs(w.mean()) < 0.01
    assert (w * w).mean() == pytest.approx(float(out["second_moment_w2"][0]), rel=0.01)
    assert (w ** 3).mean() == pytest.approx(float(out["third_moment_w3"][0]), rel=0.03)


def _chain(**kw):
    from flexpart_gpu import convection as cv
    a = dict(precip=10.0, wstar=2.4, hbl=850.0, cape=850.0, dt=600.0)
    a.update(kw)
    return cv.build_simplified_convection_chain(
        cv.SimplifiedEmanuelInputs(IFACE, a["precip"], a["wstar"], a["hbl"], a["cape"]), a["dt"])


def test_convective_mixing_matches_the_reference_chain_test(ctx):
    # tests/convection_chain.rs:54-93 and src/gpu/convection.rs:292-345
    from flexpart_gpu import convection as cv
    column, matrix = _chain(precip=12.0, wstar=2.8, hbl=900.0, cape=900.0)
    rec = _records([(0.5, 0.5, 150.0), (0.5, 0.5, 700.0), (0.5, 0.5, 1700.0), (0.5, 0.5, 3200.0)], [1, 1, 1, 0])
    rec["mass"][:, 0] = [1.0, 2.0, 3.0, 4.0]
    p = _upload(ctx, rec)
    cm = cv.dispatch_convective_mixing_gpu(ctx, p, column.level_interfaces_m, matrix)
    got = p.download()
    ref = orc.convective_mixing(rec, matrix.coefficients_column_major, IFACE)
    assert got.tobytes() == ref.tobytes()
    assert got["pos_z"][3] == 3200.0 and got["cbt"][3] == 0           # inactive: untouched
    assert np.array_equal(got["mass"], rec["mass"])
    L = matrix.level_count()
    for s in range(L):                                                 # the per-level table
        one = _records([(0.5, 0.5, float(column.level_centers_m[s]))])
        assert cm.heights()[s] == orc.convective_mixing(one, matrix.coefficients_column_major, IFACE)["pos_z"][0]


def test_convective_mixing_bit_exact_on_a_million_slots(ctx):
    from flexpart_gpu import convection as cv
    rng = np.random.default_rng(4)
    n = 1_000_003                                                      # a ragged last quad
    z = rng.uniform(-1000.0, 6000.0, n).astype(np.float32)
    z[:8] = np.float32(IFACE + [np.nan, np.inf])[:8]
    rec = _records(np.c_[np.full(n, 0.5), np.full(n, 0.5), z], (rng.random(n) > 0.25).astype(np.uint32))
    rec["pos_z"] = z
    for kw in ({}, dict(precip=0.0, wstar=0.0, cape=None), dict(dt=60.0), dict(precip=40.0, cape=3000.0)):
        _, matrix = _chain(**kw)
        p = _upload(ctx, rec)
        cm = cv.ConvectiveMixing(ctx, matrix.level_count())
        cm.set_matrix(matrix, IFACE)
        cm.apply(p)
        got = p.download()
        ref = orc.convective_mixing(rec, matrix.coefficients_column_major, IFACE)
        assert got.tobytes() == ref.tobytes(), kw


def test_convective_mixing_unsorted_interfaces_use_the_linear_scan(ctx):
    """The shader's first-match scan on interfaces that are not increasing
    (the device object accepts them, as the reference's dispatch does)."""
    from flexpart_gpu import convection as cv
    iface = [0.0, 2000.0, 1000.0, 3000.0, 2500.0, 5000.0]
    L = 5
    rng = np.random.default_rng(2)
    m = rng.uniform(0.0, 1.0, (L, L)).astype(np.float32)
    m /= m.sum(axis=1, keepdims=True, dtype=np.float32)
    m = m.astype(np.float32).reshape(-1)
    n = 100_000
    rec = _records(np.c_[np.full(n, 0.5), np.full(n, 0.5), rng.uniform(-100, 5100, n)])
    p = _upload(ctx, rec)
    cm = cv.ConvectiveMixing(ctx, L)
    try:
        cm.set_matrix(m, iface)
    except Exception as e:                                             # float32 column sums off by > 1e-4
        pytest.skip(f"random matrix rejected: {e}")
    cm.apply(p)
    assert p.download().tobytes() == orc.convective_mixing(rec, m, iface).tobytes()


def test_convection_errors(ctx):
    from flexpart_gpu import convection as cv
    from flexpart_gpu._lib import FpgError
    with pytest.raises(FpgError) as e:
        cv.ConvectiveMixing(ctx, 0)
    assert e.value.status == -3
    cm = cv.ConvectiveMixing(ctx, 5)
    bad = np.eye(5, dtype=np.float32).reshape(-1)
    bad[0] = 0.5
    with pytest.raises(FpgError) as e:
        cm.set_matrix(bad, IFACE)
    assert e.value.status == -23
    with pytest.raises(FpgError) as e:
        cm.set_matrix(np.eye(5, dtype=np.float32).reshape(-1), IFACE[:-1])
    assert e.value.status == -5
    with pytest.raises(FpgError) as e:                                 # never set
        cm.apply(_upload(ctx, _records([(0.5, 0.5, 10.0)])))
    assert e.value.status == -11
    from flexpart_gpu import cbl
    rec = _records([(0.5, 0.5, 10.0)] * 3)
    with pytest.raises(FpgError) as e:                                 # MismatchedInputLengths
        cbl.sample_cbl_vertical_velocity_gpu(ctx, _upload(ctx, rec), np.zeros(2, cbl.HANNA_PARAMS_DTYPE),
                                             cbl.sampling_inputs([0.1] * 3, [0.2] * 3, [0.3] * 3))
    assert e.value.status == -5


@pytest.mark.parametrize("n_substeps", [4, 2, 0])
def test_separated_hanna_then_langevin_equals_the_fused_kernel(ctx, n_substeps):
    """The reference's validation/backward path (hanna_params.wgsl then
    langevin.wgsl on the record buffer) against its production path (the
    fused kernel): with the records of fpg_dispatch_hanna_params the two
    give the same bits, and the same next Philox counter."""
    from flexpart_gpu import cbl
    rng = np.random.default_rng(9)
    nx, ny, n = 30, 20, 200_003
    pbl, _ = _pbl(ctx, nx, ny, rng)
    rec = _records(np.c_[rng.uniform(0, nx, n), rng.uniform(0, ny, n), rng.uniform(-5, 3000, n)],
                   (rng.random(n) > 0.1).astype(np.uint32))
    rec["turb_u"], rec["turb_v"], rec["turb_w"] = (rng.normal(0, 0.5, n).astype(np.float32) for _ in range(3))
    rec["cbt"] = rng.choice([-1, 1], n).astype(np.int32)
    key, counter = (0xDECAFBAD, 0x12345678), (0xA5A50001, 0xFACEB00C, 7, 9)
    pa, pb = _upload(ctx, rec), _upload(ctx, rec)
    na = api.langevin_fused(ctx, pa, pbl, 600.0, 2.5e-4, n_substeps, 0.01, key, counter)
    hanna = cbl.dispatch_hanna_params_gpu(ctx, pb, pbl)
    nb = cbl.update_particles_turbulence_langevin_gpu(ctx, pb, hanna, 600.0, 2.5e-4, n_substeps, 0.01, key, counter)
    assert na == nb == orc.next_counter(list(counter), n, n_substeps)
    assert pa.download().tobytes() == pb.download().tobytes()


def test_langevin_with_hanna_records_matches_the_reference_legacy_case(ctx):
    # src/gpu/langevin.rs:662-805: five particles over a 4x1 PBL (unstable,
    # neutral, stable, unstable), the last inactive; Hanna records on the
    # device, then the legacy Langevin step (dt 45 s, rho'/rho 2.5e-4, no
    # sub-steps) against the oracle's turbulence at 5e-5
    from flexpart_gpu import cbl
    from flexpart_gpu.records import StepParams
    rec = _records([(0.2, 0.0, 120.0), (1.1, 0.0, 80.0), (2.1, 0.0, 200.0), (3.0, 0.0, 300.0), (3.2, 0.0, 30.0)],
                   [1, 1, 1, 1, 0])
    rec["turb_u"] = [0.8, -0.5, 0.4, -0.2, 0.0]
    rec["turb_v"] = [-0.3, 1.1, 0.7, -0.4, 0.0]
    rec["turb_w"] = [0.1, -0.2, -1.0, 0.6, 0.0]
    ust, wst = [0.30, 0.25, 0.35, 0.28], [1.80, 0.0, 0.0, 1.60]
    hmix, oli = [900.0, 800.0, 700.0, 1000.0], [-0.02, 0.0, 0.01, -0.0125]
    pbl = api.Pbl(ctx, 4, 1)
    pbl.upload(ust, wst, hmix, oli)
    p = _upload(ctx, rec)
    hanna = cbl.compute_hanna_params_gpu(ctx, p, pbl)
    ref_h = orc.hanna_params_slots(rec, ust, wst, hmix, oli, 4, 1)
    # np.isclose: the neutral cell's L = +inf on both sides
    assert np.isclose(hanna.view(np.float32).reshape(5, 16)[:, :13], ref_h[:, :13], rtol=5e-5, atol=5e-5).all()
    key, counter = (0xDECAFBAD, 0x12345678), (0xA5A50001, 0xFACEB00C, 7, 9)
    nxt = cbl.update_particles_turbulence_langevin_gpu(ctx, p, hanna, 45.0, 2.5e-4, 0, 0.01, key, counter)
    assert nxt == orc.counter_add(list(counter), 5)
    o = orc.Pbl(4, 1)
    o.ustar[:], o.wstar[:], o.hmix[:], o.oli[:] = ust, wst, hmix, oli
    s = orc.State.from_records(rec)
    prm = StepParams.production(turb_dt_seconds=45.0, rho_grad_over_rho=2.5e-4, key=key, counter=counter)
    prm.stages, prm.n_substeps, prm.dry_mode, prm.wet_mode = 2, 0, 0, 0
    flat = {k: np.zeros((4, 1, 2), np.float32) for k in ("u0", "v0", "w0", "u1", "v1", "w1")}
    flat["heights"] = np.array([0.0, 1000.0], np.float32)             # no advection in this step
    orc.step(s, 5, flat, o, prm)
    got = p.download()
    for f in ("turb_u", "turb_v", "turb_w"):
        assert _close(got[f], getattr(s, f), 5e-5, 5e-5).all(), f
    for f in ("pos_x", "pos_y", "pos_z", "cell_x", "cell_y", "flags", "cbt"):
        assert np.array_equal(got[f], rec[f]), f                          # legacy: only the turbulence moves
    assert np.all(got[4].tobytes() == rec[4].tobytes())


def test_langevin_with_hanna_errors(ctx):
    from flexpart_gpu import cbl
    from flexpart_gpu._lib import FpgError
    rec = _records([(0.5, 0.5, 10.0)] * 3)
    p = _upload(ctx, rec)
    with pytest.raises(FpgError) as e:                                 # MismatchedInputLengths
        cbl.update_particles_turbulence_langevin_gpu(ctx, p, np.zeros(2, cbl.HANNA_PARAMS_DTYPE), 60.0, 0.0, 4,
                                                     0.01, (1, 2), (0, 0, 0, 0))
    assert e.value.status == -5
    with pytest.raises(FpgError) as e:                                 # InvalidTimeStep
        cbl.update_particles_turbulence_langevin_gpu(ctx, p, np.zeros(3, cbl.HANNA_PARAMS_DTYPE), 0.0, 0.0, 4,
                                                     0.01, (1, 2), (0, 0, 0, 0))
    assert e.value.status == -2
    # zero records: sanitize_positive gives zero T_L, hence zero turbulence (langevin.wgsl:189-238)
    nxt = cbl.update_particles_turbulence_langevin_gpu(ctx, p, np.zeros(3, cbl.HANNA_PARAMS_DTYPE), 60.0, 0.0, 0,
                                                       0.01, (1, 2), (0, 0, 0, 0))
    assert nxt == [3, 0, 0, 0]
    got = p.download()
    assert np.all(got["turb_u"] == 0) and np.all(got["turb_w"] == 0)


def test_record_pointers_must_be_16_byte_aligned(ctx):
    """The CBL and Hanna kernels move records as 16-byte vectors; a
    misaligned device pointer is refused before any launch."""
    from flexpart_gpu import cbl
    from flexpart_gpu._lib import lib
    rec = _records([(0.5, 0.5, 10.0)] * 4)
    p = _upload(ctx, rec)
    pbl = api.Pbl(ctx, 1, 1)
    pbl.upload([0.3], [1.0], [800.0], [-0.01])
    buf = api.DeviceArray(ctx, 64 * 5, np.uint8)
    off = api._vp(buf.ptr + 4)
    assert lib.fpg_dispatch_hanna_params(ctx.h, p.h, pbl.h, off, 4, None) == -1
    assert lib.fpg_cbl_sample(ctx.h, p.h, off, 4, api._vp(buf.ptr), 4, api._vp(buf.ptr), None) == -1
    k, c = api._u32arr((1, 2), 2), api._u32arr((0, 0, 0, 0), 4)
    assert lib.fpg_cbl_sample_philox(ctx.h, p.h, pbl.h, k, c, off, None) == -1
    out = cbl.sample_cbl_vertical_velocity_philox(ctx, p, pbl, (1, 2), (0, 0, 0, 0))   # aligned: fine
    assert out.size == 4


def test_edge_sizes(ctx):
    """One convection level; an empty dispatch for every entry point."""
    from flexpart_gpu import cbl
    from flexpart_gpu import convection as cv
    rec = _records([(0.5, 0.5, -20.0), (0.5, 0.5, 300.0), (0.5, 0.5, 5000.0)], [1, 1, 0])
    p = _upload(ctx, rec)
    cm = cv.ConvectiveMixing(ctx, 1)
    cm.set_matrix(np.ones(1, np.float32), [0.0, 1000.0])
    cm.apply(p)
    got = p.download()
    assert got["pos_z"].tolist() == [500.0, 500.0, 5000.0] and got["cbt"].tolist() == [0, 0, 0]
    assert got.tobytes() == orc.convective_mixing(rec, np.ones(1, np.float32), [0.0, 1000.0]).tobytes()
    empty = api.Particles(ctx, 4)
    empty.dispatch_count = 0
    cm.apply(empty)
    pbl = api.Pbl(ctx, 1, 1)
    pbl.upload([0.3], [1.0], [800.0], [-0.01])
    assert cbl.compute_hanna_params_gpu(ctx, empty, pbl).size == 0
    assert cbl.sample_cbl_vertical_velocity_philox(ctx, empty, pbl, (1, 2), (0, 0, 0, 0)).size == 0
    assert cbl.sample_cbl_vertical_velocity_gpu(ctx, empty, np.zeros(0, cbl.HANNA_PARAMS_DTYPE),
                                                np.zeros(0, cbl.CBL_INPUT_DTYPE)).size == 0
    assert cbl.update_particles_turbulence_langevin_gpu(ctx, empty, np.zeros(0, cbl.HANNA_PARAMS_DTYPE), 60.0, 0.0,
                                                        4, 0.01, (1, 2), (5, 0, 0, 0)) == [5, 0, 0, 0]
