"""Pins the C oracle to the reference's own known-answer vectors and analytic
tests (read from the reference's test sources; cited per test).  CPU only.
"""
import math

import numpy as np
import pytest

from oracle import orc


# ---- Philox (src/physics/rng.rs:171-215) -----------------------------------

def test_philox_zero_vector_matches_reference_block():
    # rng.rs:172-177
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_philox_counter_add_handles_carry():
    # rng.rs:211-215
    assert orc.counter_add([0xFFFFFFFF, 0xFFFFFFFF, 7, 9], 1) == [0, 0, 8, 9]


def test_philox_stream_uniform_mean_is_near_half():
    # rng.rs:191-208: 200k uniforms from key/counter of the test, mean within 0.01
    u, _ = orc.philox_uniforms([0xA4093822, 0x299F31D0], [0x243F6A88, 0x85A308D3, 0, 0], 50_000)
    assert np.all((u >= 0) & (u < 1))
    assert abs(float(np.mean(u.astype(np.float64))) - 0.5) < 0.01


def test_u32_to_uniform_uses_high_24_bits():
    # rng.rs:94-96
    assert orc.u32_to_uniform01(0xFFFFFFFF) == np.float32(16777215 / 16777216)
    assert orc.u32_to_uniform01(0xFF) == 0.0


def test_counter_advance_blocks_per_particle():
    # gpu/langevin_fused.rs:229-233: 1 block for n_substeps <= 2, else 2; none for 0 particles
    assert orc.next_counter([5, 0, 0, 0], 10, 4) == [25, 0, 0, 0]
    assert orc.next_counter([5, 0, 0, 0], 10, 2) == [15, 0, 0, 0]
    assert orc.next_counter([5, 0, 0, 0], 0, 4) == [5, 0, 0, 0]


# ---- Langevin (src/physics/langevin.rs:361-409) -----------------------------

def test_langevin_zero_turbulence_is_deterministic_decay():
    # langevin.rs:362-381: zeroed Hanna params except TL = 50, legacy dt = 10, zero noise
    u = orc.langevin_h(2.0, 0.0, 50.0, 10.0, 0.0)
    v = orc.langevin_h(-1.0, 0.0, 50.0, 10.0, 0.0)
    w = orc.langevin_v(0.5, 0.0, 50.0, 0.0, 10.0, 0.0, 0.0)
    assert abs(u - 1.6) < 1e-6
    assert abs(v + 0.8) < 1e-6
    assert abs(w - 0.4) < 1e-6


def test_langevin_finite_dt_bounded():
    # langevin.rs:384-409
    h = orc.hanna(0.3, 1.2, -100.0, 900.0, 120.0)
    u = orc.langevin_h(12.0, h["sigu"], h["tlu"], 180.0, 0.5)
    v = orc.langevin_h(-9.0, h["sigv"], h["tlv"], 180.0, -0.3)
    w = orc.langevin_v(6.0, h["sigw"], h["tlw"], h["dsigwdz"], 180.0, 5e-4, 0.2)
    for x in (u, v, w):
        assert math.isfinite(x) and abs(x) < 100.0


def test_box_muller_clamps_edges():
    # langevin.rs:176-182: u0 = 0 is clamped to MIN_POSITIVE, never log(0)
    a, b = orc.box_muller(0.0, 0.0)
    assert math.isfinite(a) and b == 0.0
    a, b = orc.box_muller(1.0, 1.0)
    assert math.isfinite(a) and math.isfinite(b)


# ---- Trilinear interpolation (src/physics/interpolation.rs:93-183) ---------

def _corner_field():
    u = np.zeros((2, 2, 2), np.float32)
    for i in range(2):
        for j in range(2):
            for k in range(2):
                u[i, j, k] = i + 10 * j + 100 * k
    return u, u + 1, -u


def test_trilinear_exact_corner_values():
    u, v, w = _corner_field()
    assert orc.trilinear(u, 1.0, 0.0, 1.0) == 101.0
    assert orc.trilinear(v, 1.0, 0.0, 1.0) == 102.0
    assert orc.trilinear(w, 1.0, 0.0, 1.0) == -101.0


def test_trilinear_cell_center_is_corner_average():
    u, v, w = _corner_field()
    for f in (u, v, w):
        assert abs(orc.trilinear(f, 0.5, 0.5, 0.5) - f.sum() / 8.0) < 1e-6


def test_trilinear_linear_field_is_exact():
    nx, ny, nz = 4, 3, 5
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.astype(np.float32), j.astype(np.float32), k.astype(np.float32)
    u = 2 * i + 3 * j - 0.5 * k + 7
    v = -1.25 * i + 0.75 * j + 2.5 * k - 4
    w = 0.5 * i - 2 * j + 4 * k + 1.5
    x, y, z = 2.2, 1.4, 3.1
    assert abs(orc.trilinear(u, x, y, z) - (2 * x + 3 * y - 0.5 * z + 7)) < 1e-5
    assert abs(orc.trilinear(v, x, y, z) - (-1.25 * x + 0.75 * y + 2.5 * z - 4)) < 1e-5
    assert abs(orc.trilinear(w, x, y, z) - (0.5 * x - 2 * y + 4 * z + 1.5)) < 1e-5


def test_trilinear_out_of_bounds_coordinates_are_clamped():
    u, v, w = _corner_field()
    assert orc.trilinear(u, -8.0, 99.0, 5.0) == u[0, 1, 1]
    assert orc.trilinear(v, -8.0, 99.0, 5.0) == v[0, 1, 1]
    assert orc.trilinear(w, -8.0, 99.0, 5.0) == w[0, 1, 1]


# ---- Advection (src/physics/advection.rs:282-487) ---------------------------

def _state_at(points):
    s = orc.State(len(points))
    for n, (x, y, z) in enumerate(points):
        cx, cy = math.floor(x), math.floor(y)
        s.cell_x[n], s.cell_y[n] = cx, cy
        s.pos_x[n] = np.float32(np.float32(x) - np.float32(cx))
        s.pos_y[n] = np.float32(np.float32(y) - np.float32(cy))
        s.pos_z[n] = z
        s.flags[n] = 1
    return s


def test_advection_uniform_wind_matches_analytical_solution():
    # advection.rs:282-331, tolerance 1e-5
    dt, u, v, w = np.float32(2.75), np.float32(0.8), np.float32(-0.35), np.float32(0.15)
    shape = (64, 64, 64)
    pts = [(5.25, 8.5, 6.25), (11.0, 13.125, 9.75), (23.9, 17.4, 12.1), (31.375, 4.2, 3.0)]
    s = _state_at(pts)
    orc.advect_cpu(s, np.full(shape, u, np.float32), np.full(shape, v, np.float32),
                   np.full(shape, w, np.float32), dt)
    for n, (x0, y0, z0) in enumerate(pts):
        assert abs(s.grid_x()[n] - float(np.float32(x0) + u * dt)) <= 1e-5
        assert abs(s.grid_y()[n] - float(np.float32(y0) + v * dt)) <= 1e-5
        assert abs(float(s.pos_z[n]) - float(np.float32(z0) + w * dt)) <= 1e-5
        assert abs(s.vel_u[n] - u) <= np.finfo(np.float32).eps
        assert abs(s.vel_v[n] - v) <= np.finfo(np.float32).eps
        assert abs(s.vel_w[n] - w) <= np.finfo(np.float32).eps


def test_petterssen_linear_shear_is_more_accurate_than_euler():
    # advection.rs:333-364
    a, dt, x0 = np.float32(0.2), np.float32(1.0), 2.5
    u = np.zeros((64, 4, 4), np.float32)
    u[:] = (a * np.arange(64, dtype=np.float32))[:, None, None]
    zero = np.zeros_like(u)
    s = _state_at([(x0, 1.0, 1.0)])
    orc.advect_cpu(s, u, zero, zero, dt)
    euler_x = x0 + orc.trilinear(u, x0, 1.0, 1.0) * dt
    exact = x0 * math.exp(a * dt)
    assert abs(s.grid_x()[0] - exact) < abs(euler_x - exact)


def test_advection_clamps_out_of_domain_position_stably():
    # advection.rs:366-380
    shape = (3, 3, 3)
    s = _state_at([(1.8, 0.2, 1.0)])
    orc.advect_cpu(s, np.full(shape, 10, np.float32), np.full(shape, -10, np.float32),
                   np.full(shape, 10, np.float32), 1.0)
    assert (s.cell_x[0], s.pos_x[0], s.cell_y[0], s.pos_y[0], s.pos_z[0]) == (2, 0.0, 0, 0.0, 2.0)


def _shear_field(n, u_ref, v_ref, w_c, du, dv):
    # wind/synthetic.rs:101-129 with heights = level index
    k = np.arange(n, dtype=np.float32)
    u = np.broadcast_to((np.float32(u_ref) + np.float32(du) * k)[None, None, :], (n, n, n))
    v = np.broadcast_to((np.float32(v_ref) + np.float32(dv) * k)[None, None, :], (n, n, n))
    w = np.full((n, n, n), w_c, np.float32)
    return np.ascontiguousarray(u), np.ascontiguousarray(v), w


def _analytic(x0, y0, z0, t, u_ref, v_ref, w_c, du, dv):
    # advection.rs:260-280
    u_t0 = u_ref + du * z0
    v_t0 = v_ref + dv * z0
    return (x0 + u_t0 * t + 0.5 * du * w_c * t * t, y0 + v_t0 * t + 0.5 * dv * w_c * t * t,
            z0 + w_c * t)


def test_petterssen_linear_shear_matches_analytical_single_step():
    # advection.rs:382-432, tolerance 1e-5
    u, v, w = _shear_field(96, 1.2, -0.35, 0.2, 0.04, -0.015)
    s = _state_at([(10.25, 11.75, 5.4)])
    orc.advect_cpu(s, u, v, w, 0.6)
    ex = _analytic(10.25, 11.75, 5.4, 0.6, 1.2, -0.35, 0.2, 0.04, -0.015)
    assert abs(s.grid_x()[0] - ex[0]) <= 1e-5
    assert abs(s.grid_y()[0] - ex[1]) <= 1e-5
    assert abs(s.pos_z[0] - ex[2]) <= 1e-5


def test_petterssen_linear_shear_matches_analytical_multi_step():
    # advection.rs:434-487, 20 steps, tolerance 2e-4
    u, v, w = _shear_field(128, 0.8, 0.5, 0.3, 0.03, -0.02)
    s = _state_at([(8.125, 9.625, 6.5)])
    for _ in range(20):
        orc.advect_cpu(s, u, v, w, 0.25)
    ex = _analytic(8.125, 9.625, 6.5, 5.0, 0.8, 0.5, 0.3, 0.03, -0.02)
    assert abs(s.grid_x()[0] - ex[0]) <= 2e-4
    assert abs(s.grid_y()[0] - ex[1]) <= 2e-4
    assert abs(s.pos_z[0] - ex[2]) <= 2e-4


# ---- Hanna (src/physics/hanna.rs:227-519) ----------------------------------

def test_hanna_neutral_sigmas_decrease_with_height():
    lo = orc.hanna(0.4, 0.0, 2000.0, 1000.0, 20.0)
    hi = orc.hanna(0.4, 0.0, 2000.0, 1000.0, 600.0)
    assert hi["sigu"] < lo["sigu"] and hi["sigw"] < lo["sigw"]


def test_hanna_stable_sigma_u_decreases_with_height():
    lo = orc.hanna(0.35, 0.0, 100.0, 1000.0, 50.0)
    hi = orc.hanna(0.35, 0.0, 100.0, 1000.0, 500.0)
    assert hi["sigu"] < lo["sigu"]


def test_hanna_unstable_vs_stable_vertical_sigma_difference():
    st = orc.hanna(0.3, 1.5, 120.0, 1000.0, 100.0)
    un = orc.hanna(0.3, 1.5, -120.0, 1000.0, 100.0)
    assert un["sigw"] > st["sigw"] and un["tlu"] >= st["tlu"]


def test_hanna_no_nan_or_inf_for_realistic_ranges():
    for ust in (0.05, 0.2, 0.6):
        for wst in (0.0, 0.8, 2.5):
            for ol in (-500.0, -80.0, 80.0, 500.0, 2.0e6):
                for h in (100.0, 800.0, 2500.0):
                    for z in (0.0, 5.0, 50.0, 200.0, 700.0, 2000.0):
                        for dtype in (np.float32, np.float64):
                            p = orc.hanna(ust, wst, ol, h, z, dtype)
                            assert all(math.isfinite(x) for x in p.values())
                            assert p["sigu"] > 0 and p["sigv"] > 0 and p["sigw"] > 0
                            assert p["tlu"] >= 10 and p["tlv"] >= 10 and p["tlw"] >= 30


def test_hanna_from_pbl_matches_direct_call():
    # hanna.rs:326-356: oli -0.02 -> L = -50
    ol = orc.obukhov_from_inverse(-0.02)
    a = orc.hanna(0.25, 1.8, ol, 900.0, 120.0)
    b = orc.hanna(0.25, 1.8, -50.0, 900.0, 120.0)
    for k in a:
        assert abs(a[k] - b[k]) < 1e-6


@pytest.mark.parametrize(
    "inp,su,sw,tol",
    [
        ((0.30, 0.0, 120.0, 1000.0, 100.0), 1.83, 1.20, 0.20),   # stable, hanna.rs:361-373
        ((0.28, 0.0, 150.0, 1000.0, 500.0), 1.04, 0.66, 0.22),   # stable, :374-386
        ((0.30, 0.0, 5000.0, 1000.0, 50.0), 1.93, 1.29, 0.16),   # neutral, :415-427
        ((0.32, 0.0, 5000.0, 1000.0, 600.0), 1.17, 0.93, 0.20),  # neutral, :428-440
        ((0.30, 2.0, -80.0, 1000.0, 100.0), 2.66, 3.51, 0.22),   # unstable, :469-481
        ((0.30, 2.0, -80.0, 1000.0, 600.0), 2.66, 4.32, 0.22),   # unstable, :482-494
    ],
)
def test_hanna_table_style_ratios(inp, su, sw, tol):
    p = orc.hanna(*inp)
    assert abs(p["sigu"] / p["ust"] - su) <= su * tol
    assert abs(p["sigw"] / p["ust"] - sw) <= sw * tol


def test_hanna_short_matches_full_vertical_parameters():
    # langevin_fused.wgsl:296-344 restates the vertical half of compute_hanna
    for inp in [(0.3, 1.2, -100.0, 900.0, 120.0), (0.3, 0.0, 120.0, 1000.0, 100.0),
                (0.3, 0.0, float("inf"), 1000.0, 50.0), (0.2, 2.0, -30.0, 800.0, 500.0)]:
        full = orc.hanna(*inp)
        short = orc.hanna_short_w(*inp)
        assert short == (full["sigw"], full["dsigwdz"], full["tlw"])


# ---- Deposition (tests/integration/deposition_decay.rs) --------------------

def test_deposition_mass_evolution_matches_analytical_exponential_decay():
    # deposition_decay.rs:11-27,222-270: 12 steps of 60 s, vdep 0.024, lambda 1.6e-3,
    # fraction 1, z = 5 m, href 15, CPU tolerance 2e-6
    m0 = np.array([1.0, 0.4, 0.2, 0.1], np.float32)
    dry_rate = float(np.float32(0.024) / (np.float32(2.0) * np.float32(15.0)))
    wet_rate = float(np.float32(1.6e-3))
    md, mw, mc = m0.copy(), m0.copy(), m0.copy()
    for step in range(1, 13):
        sd = np.float32(orc.dry_survival(0.024, 60.0, 15.0))
        pw = np.float32(orc.wet_probability(1.6e-3, 60.0, 1.0))
        md = (md * sd).astype(np.float32)
        mw = (mw * (np.float32(1) - pw)).astype(np.float32)
        mc = ((mc * sd).astype(np.float32) * (np.float32(1) - pw)).astype(np.float32)
        t = step * 60.0
        tot0 = float(m0.astype(np.float64).sum())
        for sim, rate in ((md, dry_rate), (mw, wet_rate), (mc, dry_rate + wet_rate)):
            exp = tot0 * math.exp(-rate * t)
            assert abs(float(sim.astype(np.float64).sum()) - exp) <= max(2e-6, 2e-6 * exp)


# ---- Gridding (tests/integration/scientific_invariants.rs:49-164) ----------

def test_gridding_matches_reference_cpu_case_with_outheights():
    pts = [(2, 3, 50.0, 1.5), (2, 3, 150.0, 0.8), (5, 1, 600.0, 2.0), (7, 5, 999.0, 0.3),
           (0, 0, 10.0, 4.0), (1, 1, 80.0, 9.9)]
    s = orc.State(len(pts))
    for n, (cx, cy, z, m) in enumerate(pts):
        s.cell_x[n], s.cell_y[n], s.pos_x[n], s.pos_y[n], s.pos_z[n] = cx, cy, 0.3, 0.6, z
        s.mass[0, n] = m
        s.flags[n] = 0 if n == 5 else 1
    shape = (8, 6, 3)
    counts, mass_scaled, _ = orc.grid(s, len(pts), 0, 1e6, [100.0, 500.0, 1000.0], shape)
    # the reference test's CPU binning (scientific_invariants.rs:49-85)
    ref_counts = np.zeros(8 * 6 * 3, np.uint32)
    ref_mass = np.zeros(8 * 6 * 3, np.float32)
    for n, (cx, cy, z, m) in enumerate(pts):
        if n == 5:
            continue
        iz = next((k for k, hgt in enumerate([100.0, 500.0, 1000.0]) if z <= hgt), 2)
        flat = (cx * 6 + cy) * 3 + iz
        ref_counts[flat] += 1
        ref_mass[flat] += np.float32(round(np.float32(m) * np.float32(1e6))) / np.float32(1e6)
    assert np.array_equal(counts, ref_counts)
    assert np.all(np.abs(mass_scaled.astype(np.float32) / np.float32(1e6) - ref_mass) < 1e-4)
    assert counts.sum() == 5


def test_gridding_levels_top_bin_and_legacy_floor():
    # concentration_gridding.wgsl:304-315: above the top height goes to the top level;
    # zero outheights use floor(z) clamped
    assert orc.level_of(5000.0, [100.0, 500.0, 1000.0]) == 2
    assert orc.level_of(100.0, [100.0, 500.0, 1000.0]) == 0
    assert orc.level_of(2.7, [0.0, 0.0, 0.0]) == 2
    assert orc.level_of(-3.0, [0.0, 0.0, 0.0]) == 0
    assert orc.level_of(1.2, [0.0, 0.0, 0.0]) == 1


# ---- Compaction (src/gpu/compaction.rs:624-740) ----------------------------

@pytest.mark.parametrize(
    "n,inactive",
    [(1000, lambda i: i % 3 == 0), (512, lambda i: False), (256, lambda i: True),
     (100, lambda i: i != 42), (300, lambda i: i % 5 == 0), (1000, lambda i: i % 2 == 0)],
)
def test_compaction_sets(n, inactive):
    flags = np.array([0 if inactive(i) else 1 for i in range(n)], np.uint32)
    count, idx = orc.compaction_indices(flags)
    expected = [i for i in range(n) if not inactive(i)]
    assert count == len(expected)
    assert set(idx.tolist()) == set(expected)       # the reference's set check
    assert idx.tolist() == expected                  # and the order is stable


# ---- Time bookkeeping ------------------------------------------------------

def test_interpolation_alpha_sequence():
    # tests/forward_timeloop.rs:119-126 with bracket [t0, t0+2]
    for k, a in enumerate([0.0, 0.5, 1.0]):
        st, v = orc.interpolation_alpha(100, 102, 100 + k)
        assert st == 0 and abs(v - a) < 1e-6
    assert orc.interpolation_alpha(100, 100, 100)[0] == -12
    assert orc.interpolation_alpha(100, 102, 200, clamp=False)[0] == -13
    assert orc.interpolation_alpha(100, 102, 200, clamp=True)[1] == 1.0


def test_release_counts_and_bounds():
    # release/mod.rs:391-455: 12 particles over [01:00, 02:00]
    st, start = orc.parse_timestamp("20240101010000")
    _, end = orc.parse_timestamp("20240101020000")
    assert st == 0
    t = lambda s: orc.parse_timestamp(s)[1]
    assert orc.target_emitted_count(12, start, end, t("20240101005959"), 0) == 0
    assert orc.target_emitted_count(12, start, end, t("20240101020001"), 0) == 0
    n1 = orc.target_emitted_count(12, start, end, t("20240101011500"), 0)
    n2 = orc.target_emitted_count(12, start, end, t("20240101014500"), n1)
    n3 = orc.target_emitted_count(12, start, end, t("20240101020000"), n2)
    assert (n1, n2 - n1, n3 - n2) == (3, 6, 3)
    bounds = (10.0, 12.0, 45.0, 46.0, 100.0, 200.0)
    domain = (0.0, 0.0, 1.0, 1.0, 40, 80)
    for i in range(12):
        lon, lat, z = orc.sample_stratified(bounds, i, 12)
        stt, cx, cy, fx, fy = orc.geo_to_relative(lon, lat, domain)
        assert stt == 0
        assert 10.0 <= cx + fx <= 12.0 and 45.0 <= cy + fy <= 46.0 and 100.0 <= z <= 200.0


def test_timestamp_epoch():
    # fortran-validation.rs:207: 2024-01-01 00:00:00 UTC = 1704067200
    assert orc.parse_timestamp("20240101000000") == (0, 1704067200)
