"""CBL skewed PDF and convective mixing on the CPU.

* The oracle's CBL restatement is pinned to the reference's own tests
  (physics/cbl.rs:333-474): moment reconstruction, deterministic Philox
  sampling that reproduces the target moments, the symmetric fallback, the
  sign of branch-constrained samples, a positive density.
* The library's host-side convection builder (C++, fpg_convection_build_chain)
  is held to the reference's convection tests (physics/convection.rs:492-625,
  tests/convection_chain.rs:26-61) and must equal the oracle's restatement
  bit for bit; its errors carry the reference's error kinds.
No GPU: the builder is host code, the sampler here is the oracle's.
"""
import numpy as np
import pytest

from oracle import orc

IFACE = [0.0, 400.0, 1000.0, 2000.0, 3500.0, 5000.0]


# ---- physics/cbl.rs tests ---------------------------------------------------

def test_cbl_bigaussian_reconstructs_target_moments():
    # cbl.rs:339-374
    pdf = orc.cbl_pdf(180.0, 1200.0, 2.2, 1.1, -80.0)
    rec = orc.cbl_reconstruct_moments(pdf)
    assert 0.0 < pdf[0] < 1.0 and 0.0 < pdf[3] < 1.0
    assert pdf[2] > 0.0 and pdf[5] > 0.0
    assert rec[0] == pytest.approx(pdf[6], rel=2e-4, abs=2e-4)
    assert rec[1] == pytest.approx(pdf[7], rel=5e-4, abs=5e-4)


def test_cbl_sampling_is_deterministic_and_matches_moments():
    # cbl.rs:376-420: 100 000 draws from key 0xCAFEBABE/0x12345678, counter 7, 11, 13, 17
    pdf = orc.cbl_pdf(200.0, 1400.0, 2.4, 1.2, -90.0)
    key, ctr = [0xCAFEBABE, 0x12345678], [7, 11, 13, 17]
    a = orc.cbl_sample_stream(pdf, key, ctr, 100_000)
    b = orc.cbl_sample_stream(pdf, key, ctr, 100_000)
    assert a.tobytes() == b.tobytes()
    w = a.astype(np.float64)
    assert abs(w.mean()) < 0.03
    assert np.float32((w * w).mean()) == pytest.approx(pdf[6], rel=0.05, abs=0.05)
    assert np.float32((w ** 3).mean()) == pytest.approx(pdf[7], rel=0.12, abs=0.12)


def test_cbl_neutral_or_zero_skew_falls_back_to_symmetric_pdf():
    # cbl.rs:422-437
    pdf = orc.cbl_pdf(100.0, 1000.0, 0.0, 0.9, 1.0e6)
    for got, want in zip(pdf[:6], [0.5, 0.0, 0.9, 0.5, 0.0, 0.9]):
        assert got == pytest.approx(want, abs=1e-6)


def test_cbl_branch_constrained_sampling_preserves_sign():
    # cbl.rs:439-457
    pdf = orc.cbl_pdf(300.0, 1200.0, 1.8, 1.0, -120.0)
    assert orc.cbl_branch_constrained(pdf, "updraft", 0.2, 0.4, 1) >= 0.0
    assert orc.cbl_branch_constrained(pdf, "downdraft", 0.2, 0.4, 1) <= 0.0
    assert orc.cbl_branch_constrained(pdf, "updraft", 0.2, 0.4, -1) <= 0.0
    # infer_cbl_branch (cbl.rs:300-309): signum * direction >= 0 is updraft
    assert orc.cbl_infer_branch(0.5, 1) == "updraft"
    assert orc.cbl_infer_branch(-0.5, 1) == "downdraft"
    assert orc.cbl_infer_branch(-0.5, -1) == "updraft"
    assert orc.cbl_infer_branch(0.0, 1) == "updraft"
    assert orc.cbl_infer_branch(-0.0, 1) == "downdraft"


def test_cbl_pdf_probability_is_positive():
    # cbl.rs:459-473
    pdf = orc.cbl_pdf(150.0, 1000.0, 2.0, 1.0, -70.0)
    for w in (-5.0, -2.0, -1.0, 0.0, 1.0, 3.0, 5.0):
        assert orc.cbl_probability_density(pdf, w) >= 0.0


def test_cbl_transition_factor_edges():
    # cbl.rs:109-124: non-finite or zero inputs give 1; -h/L >= 15 gives 1;
    # -h/L = -10 gives sin(0)*0.5 + 0.5 = 0.5
    assert orc.cbl_transition_factor(float("inf"), -50.0) == 1.0
    assert orc.cbl_transition_factor(1000.0, 0.0) == 1.0
    assert orc.cbl_transition_factor(1500.0, -100.0) == 1.0
    assert orc.cbl_transition_factor(1000.0, 100.0) == pytest.approx(0.5, abs=1e-6)


# ---- physics/convection.rs tests, on the library's host builder -----------------

def _chain(precip=10.0, wstar=2.5, hbl=900.0, cape=None, dt=600.0, iface=IFACE):
    from flexpart_gpu import convection as cv
    return cv.build_simplified_convection_chain(
        cv.SimplifiedEmanuelInputs(list(iface), precip, wstar, hbl, cape), dt)


def test_simplified_emanuel_returns_inactive_column_for_weak_forcing():
    # convection.rs:504-519
    column, matrix = _chain(precip=0.0, wstar=0.0)
    assert not column.is_active
    assert np.all(column.mass_flux_profile_kg_m2_s == 0.0)
    assert np.all(column.detrainment_weights == 0.0)
    L = matrix.level_count()
    assert np.array_equal(matrix.coefficients_column_major.reshape(L, L), np.eye(L, dtype=np.float32))


def test_redistribution_matrix_is_column_stochastic():
    # convection.rs:521-537
    column, matrix = _chain()
    assert column.is_active and matrix.mixing_fraction > 0.0
    L = matrix.level_count()
    for s in range(L):
        col = [matrix.coefficient(d, s) for d in range(L)]
        assert min(col) >= -1e-6
        assert np.float32(sum(np.float32(c) for c in col)) == pytest.approx(1.0, rel=1e-5, abs=1e-5)


def test_redistribution_application_conserves_total_mass():
    # convection.rs:539-555 and tests/convection_chain.rs:26-52
    from flexpart_gpu import convection as cv
    for kw, src in (({}, [12.0, 5.0, 2.0, 0.8, 0.1]),
                    (dict(precip=10.0, wstar=2.4, hbl=850.0, cape=850.0), [16.0, 5.0, 1.5, 0.4, 0.1])):
        _, matrix = _chain(**kw)
        dst = cv.apply_redistribution_matrix(matrix, src)
        assert float(np.float32(np.sum(dst, dtype=np.float32))) == pytest.approx(
            float(np.sum(np.float32(src))), rel=1e-5, abs=1e-5)
        if kw:
            assert dst[2] > src[2] and dst[2:].sum() > sum(src[2:])


def test_flexpart_style_reference_behavior_lifts_bottom_heavy_profile():
    # convection.rs:557-567
    from flexpart_gpu import convection as cv
    _, matrix = _chain(dt=900.0)
    src = [20.0, 5.0, 1.0, 0.2, 0.1]
    dst = cv.apply_redistribution_matrix(matrix, src)
    assert dst[2] > src[2] and dst[3] > src[3]


def test_cpu_particle_mixing_moves_particles_to_expected_height():
    # convection.rs:569-624, on the oracle's particle application
    from flexpart_gpu.records import PARTICLE_DTYPE
    column, matrix = _chain()
    rec = np.zeros(2, PARTICLE_DTYPE)
    rec["flags"] = 1
    rec["pos_z"] = [200.0, 1400.0]
    out = orc.convective_mixing(rec, matrix.coefficients_column_major, IFACE)
    L = matrix.level_count()
    m = matrix.coefficients_column_major.reshape(L, L)
    s = orc.level_index_from_height(IFACE, 200.0)
    w = np.maximum(m[s], 0.0)
    expected = np.float32(0.0)
    for d in range(L):
        expected = np.float32(expected + np.float32(w[d] * column.level_centers_m[d]))
    expected = expected / np.float32(w.sum(dtype=np.float32))
    assert out["pos_z"][0] == pytest.approx(expected, rel=1e-6, abs=1e-6)
    assert list(out["cbt"]) == [0, 2]


@pytest.mark.parametrize("kw", [
    {}, dict(precip=12.0, wstar=2.8, hbl=900.0, cape=900.0), dict(precip=8.0, wstar=2.0, hbl=800.0, cape=600.0),
    dict(precip=0.06, wstar=0.1, hbl=100.0), dict(precip=50.0, wstar=4.0, hbl=3000.0, dt=60.0),
    dict(precip=10.0, wstar=2.5, hbl=900.0, cape=5.0, dt=3600.0),
])
def test_host_builder_equals_the_oracle_bit_for_bit(kw):
    kw = dict(dict(precip=10.0, wstar=2.5, hbl=900.0, cape=None, dt=600.0), **kw)
    column, matrix = _chain(**kw)
    st, m, det, info = orc.convection_chain(IFACE, kw["precip"], kw["wstar"], kw["hbl"], kw["cape"], kw["dt"])
    assert st == 0
    assert matrix.coefficients_column_major.tobytes() == m.tobytes()
    assert column.detrainment_weights.tobytes() == det.tobytes()
    assert column.is_active == bool(info["is_active"])
    assert np.float32(column.cape_j_kg) == np.float32(info["cape_j_kg"])
    assert (column.cloud_base_level, column.cloud_top_level) == (info["cloud_base_level"], info["cloud_top_level"])
    assert np.float32(matrix.mixing_fraction) == np.float32(info["mixing_fraction"])


def test_host_builder_errors_carry_the_reference_error_kinds():
    from flexpart_gpu._lib import FpgError
    cases = [(dict(iface=[0.0]), -24), (dict(iface=[0.0, 400.0, 400.0]), -25),
             (dict(iface=[0.0, float("nan")]), -25), (dict(hbl=-1.0), -26), (dict(hbl=float("inf")), -26),
             (dict(dt=0.0), -2), (dict(dt=float("nan")), -2)]
    for kw, status in cases:
        with pytest.raises(FpgError) as e:
            _chain(**kw)
        assert e.value.status == status, kw
        ref = orc.convection_chain(kw.get("iface", IFACE), 10.0, 2.5, kw.get("hbl", 900.0), None, kw.get("dt", 600.0))
        assert ref[0] == status, kw


def test_level_index_from_height_matches_the_oracle():
    from flexpart_gpu import convection as cv
    rng = np.random.default_rng(3)
    for z in np.concatenate([rng.uniform(-500, 6000, 2000).astype(np.float32),
                             np.float32(IFACE), np.float32([np.nan, np.inf, -np.inf])]):
        assert cv.level_index_from_height(IFACE, float(z)) == orc.level_index_from_height(IFACE, float(z))
    assert cv.level_index_from_height(IFACE, 5000.0) == 4          # the top interface is in the top level
    assert cv.level_index_from_height([0.0], 10.0) == 0
