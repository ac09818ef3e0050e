"""The source inversion's forward/backward pair (include/fpg_adjoint.h).

* The inversion's forward is the batched production step: its particles are
  bit-identical to a plain batch run of the same sources.
* The gradient does not depend on the checkpoint interval K, nor on
  recording the tape in the forward (K = 0) instead of recomputing it.
* Gradients against central finite differences of the device forward
  (FP32, fixed Philox counters): mass exactly (the loss is quadratic in the
  masses), positions and wind bias on a short horizon with steps where the
  FP32 differences converge.
* Gradients against the FP64 reference gradient: central differences of the
  FP64 restatement of the same forward map (oracle/inverse.py) with steps
  of 1e-9 relative (1e-8 m/s for the bias), for every parameter type.
The reference has no adjoint, so there is no reference vector to pin; the
FP64 restatement is the oracle ("parity vs restated forward map").
"""
import numpy as np
import pytest

from flexpart_gpu import synthetic

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")
adj = pytest.importorskip("flexpart_gpu.adjoint")
bt = pytest.importorskip("flexpart_gpu.batch")


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def _problem(hours, smooth, n_particles=16_000, n_sources=4, K=3):
    inv = synthetic.config3(n_particles=n_particles, n_sources=n_sources, n_receptors=10, hours=hours, smooth=smooth)
    spec = inv.ensemble.met
    # every cell of the lowest layer observed, sampled every step
    inv.receptors = [(0, i, j) for i in range(spec.nx) for j in range(spec.ny)]
    inv.sample_every = 1
    inv.checkpoint_every = K
    for s in inv.ensemble.sources:
        s.start = inv.ensemble.start
        s.end = s.start + 3600
    return inv


def _problem_c3(hours=4, n_particles=32_000, K=8):
    """The source inversion's own shape: 16 sources released over 6 h from a
    step in the first half of the run, 200 random receptor cells of the
    lowest layer, full physics (PBL per cell, dry deposition), checkpoints
    every K steps; fewer particles and a shorter horizon than the 1 M-particle
    24 h run, so that central differences of the FP64 map stay affordable and
    no particle leaves the linear range of the steps.  Receptors are sampled
    every step."""
    inv = synthetic.config3(n_particles=n_particles, n_sources=16, n_receptors=200, hours=hours)
    inv.sample_every = 1
    inv.checkpoint_every = K
    return inv


def _obs(sim, seed=1):
    rng = np.random.default_rng(seed)
    return sim * (1.0 + 0.3 * rng.standard_normal(sim.size))


def _top_bias(g, per_comp=2):
    flat = g.reshape(-1)
    out = []
    for c in range(3):
        comp = np.abs(flat[c::3])
        out += [3 * int(n) + c for n in np.argsort(comp)[::-1][:per_comp]]
    return out


def _assert_same_gradient(g, ref):
    # only the order of the device's gradient sums differs: double-precision
    # sums for the sources, a CTA's float sums per node for the wind bias
    np.testing.assert_allclose(g["mass"], ref["mass"], rtol=1e-9, atol=0)
    np.testing.assert_allclose(g["position"], ref["position"], rtol=1e-9, atol=1e-12)
    gb, rb = g["wind_bias"].astype(np.float64), ref["wind_bias"].astype(np.float64)
    assert np.linalg.norm(gb - rb) <= 1e-5 * np.linalg.norm(rb)


def test_inversion_forward_is_the_batched_step(ctx):
    inv = _problem(3, smooth=False)
    model = adj.SourceInversion(ctx, inv)
    model.forward(model.mass0, model.position0)
    from flexpart_gpu._lib import lib
    A = bt._ParticlesView(ctx, lib.fpg_batch_particles(lib.fpg_inverse_batch(model.h))).download()
    ens = inv.ensemble
    b = bt.Batch(ctx, bt.ensemble_config(ens), bt.ensemble_scenarios(ens), (ens.met.nx, ens.met.ny, ens.met.nz),
                 synthetic.level_heights(ens.met.nz, ens.met.top_m))
    for k, f in enumerate(model.frames):
        b.upload_frame(k, f, None)
    b.run(ens.n_steps)
    assert A.tobytes() == b.particles.download().tobytes()


def test_gradient_does_not_depend_on_the_checkpoint_interval(ctx):
    grads = []
    for K in (0, 1, 4, 1000):
        inv = _problem(3, smooth=False, K=K)
        model = adj.SourceInversion(ctx, inv)
        sim = model.forward(model.mass0, model.position0)
        _, d = adj.misfit(sim, _obs(sim))
        grads.append(model.backward(d))
        del model
    for g in grads[1:]:
        _assert_same_gradient(g, grads[0])


def test_gradient_across_brackets_checkpoints_and_a_repeated_backward(ctx):
    """7 h (29 steps) spans three met brackets, so the reverse sweep repacks
    the bracket where it changes (and only there).  The tape recorded in the
    forward (K = 0); checkpoints every 2 and 5 steps; the same with the last
    3 / 2 windows taped in the forward instead of recomputed; every window
    taped (W above the window count) — all give the same gradient, and a
    second backward over a tape recorded entirely in the forward repeats it."""
    grads = []
    for K, W in ((0, 0), (2, 0), (5, 0), (2, 3), (5, 2), (4, 100)):
        inv = _problem(7, smooth=False, K=K)
        inv.tape_tail_windows = W
        model = adj.SourceInversion(ctx, inv)
        sim = model.forward(model.mass0, model.position0)
        _, d = adj.misfit(sim, _obs(sim))
        grads.append(model.backward(d))
        if K == 0 or W == 100:
            _assert_same_gradient(model.backward(d), grads[-1])
        del model
    for g in grads[1:]:
        _assert_same_gradient(g, grads[0])


def test_mass_gradient_matches_device_finite_differences(ctx):
    inv = _problem(6, smooth=False)
    model = adj.SourceInversion(ctx, inv)
    sim = model.forward(model.mass0, model.position0)
    obs = _obs(sim)
    _, d = adj.misfit(sim, obs)
    g = model.backward(d, want_bias=False)
    m0 = model.mass0
    for s in range(len(m0)):
        h = 1e-3 * m0[s]
        mp, mm = m0.copy(), m0.copy()
        mp[s] += h
        mm[s] -= h
        fd = (adj.misfit(model.forward(mp), obs)[0] - adj.misfit(model.forward(mm), obs)[0]) / (2 * h)
        assert abs(g["mass"][s] - fd) <= 1e-4 * abs(fd), (s, g["mass"][s], fd)


def test_short_horizon_gradients_match_device_finite_differences(ctx):
    """1 h, uniform PBL, no deposition: positions (step 1e-4 relative) and
    horizontal wind bias (5e-3 m/s, 1e-3 of the 5 m/s mean wind) against
    FP32 central differences of the device forward.  The vertical bias is
    checked against the FP64 reference only: FP32 differences of the
    sub-stepped vertical Langevin chain do not converge at any step (large
    steps leave the linear range, small ones hit f32 rounding)."""
    inv = _problem(1, smooth=True, n_particles=32_000)
    model = adj.SourceInversion(ctx, inv)
    sim = model.forward(model.mass0, model.position0)
    obs = _obs(sim)
    _, d = adj.misfit(sim, obs)
    g = model.backward(d)
    m0, p0 = model.mass0, model.position0

    def loss(p=p0, b=None):
        return adj.misfit(model.forward(m0, p, b), obs)[0]

    errs = []
    for s in range(2):
        for c in range(3):
            h = 1e-4 * abs(p0[s, c])
            pp, pm = p0.copy(), p0.copy()
            pp[s, c] += h
            pm[s, c] -= h
            fd = (loss(p=pp) - loss(p=pm)) / (2 * h)
            errs.append(("pos", s, c, g["position"][s, c], fd))
    gb = g["wind_bias"].reshape(-1)
    for i in [i for i in _top_bias(gb, per_comp=3) if i % 3 < 2]:
        h = 5e-3
        b = np.zeros(gb.size, np.float32)
        b[i] = h
        lp = loss(b=b)
        b[i] = -h
        lm = loss(b=b)
        errs.append(("bias", i, i % 3, gb[i], (lp - lm) / (2 * h)))
    for kind, a, c, ga, fd in errs:
        print(f"{kind} {a} {c} adjoint {ga:.6e} fd {fd:.6e}")
    # the gradient vectors agree to 2e-2
    for kind in ("pos", "bias"):
        ga = np.array([e[3] for e in errs if e[0] == kind])
        fd = np.array([e[4] for e in errs if e[0] == kind])
        assert np.linalg.norm(ga - fd) <= 2e-2 * np.linalg.norm(fd), kind


@pytest.mark.parametrize("hours,smooth,shape", [(1, True, "grid"), (3, True, "grid"), (3, False, "grid"),
                                                (4, False, "c3")])
def test_gradients_match_the_fp64_reference_gradient(ctx, hours, smooth, shape):
    """Every gradient type within 1e-3 relative (in norm) of the FP64
    reference gradient: all masses, all positions, and 40 wind-bias entries
    (the 10 largest of each component and 10 drawn at random among the
    non-zero ones)."""
    from oracle.inverse import OracleInversion

    inv = _problem(hours, smooth) if shape == "grid" else _problem_c3(hours)
    model = adj.SourceInversion(ctx, inv)
    sim = model.forward(model.mass0, model.position0)
    obs = _obs(sim)
    _, d = adj.misfit(sim, obs)
    g = model.backward(d)
    o = OracleInversion(inv, model.frames)
    m0, p0 = model.mass0, model.position0
    sim64 = o.forward(m0, p0)
    # the FP32 device forward stays close to the FP64 map
    assert np.linalg.norm(sim - sim64) <= 1e-3 * np.linalg.norm(sim64)

    def loss(m=m0, p=p0, b=None):
        return float(np.sum((o.forward(m, p, b) - obs) ** 2))

    # steps of 1e-9 (positions, masses) and 1e-8 m/s (bias) in double: small
    # enough that no particle crosses a nearest-cell or branch boundary
    # between the two evaluations, large enough for FP64 rounding
    ref_m = []
    for s in range(len(m0)):
        h = 1e-9 * m0[s]
        mp, mm = m0.copy(), m0.copy()
        mp[s] += h
        mm[s] -= h
        ref_m.append((loss(m=mp) - loss(m=mm)) / (2 * h))
    ref_p = np.zeros_like(p0)
    for s in range(len(m0)):
        for c in range(3):
            h = 1e-9 * abs(p0[s, c])
            pp, pm = p0.copy(), p0.copy()
            pp[s, c] += h
            pm[s, c] -= h
            ref_p[s, c] = (loss(p=pp) - loss(p=pm)) / (2 * h)
    gb = g["wind_bias"].reshape(-1)
    idx = _top_bias(gb, per_comp=10)
    rest = np.setdiff1d(np.flatnonzero(gb != 0.0), idx)
    idx += [int(i) for i in np.random.default_rng(7).choice(rest, min(10, len(rest)), replace=False)]
    ref_b = []
    for i in idx:
        b = np.zeros(gb.size)
        b[i] = 1e-8
        lp = loss(b=b)
        b[i] = -1e-8
        ref_b.append((lp - loss(b=b)) / 2e-8)
    ref_m, ref_b = np.array(ref_m), np.array(ref_b)
    e_m = np.linalg.norm(g["mass"] - ref_m) / np.linalg.norm(ref_m)
    e_p = np.linalg.norm(g["position"] - ref_p) / np.linalg.norm(ref_p)
    e_b = np.linalg.norm(gb[idx] - ref_b) / np.linalg.norm(ref_b)
    print(f"{shape} hours {hours} smooth {smooth}: rel error mass {e_m:.2e} position {e_p:.2e} bias {e_b:.2e} "
          f"({len(idx)} bias entries)")
    print("position adjoint", g["position"].ravel(), "fp64", ref_p.ravel())
    print("bias adjoint", gb[idx], "fp64", ref_b)
    assert e_m <= 1e-3
    assert e_p <= 1e-3
    assert e_b <= 1e-3
