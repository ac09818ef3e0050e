#!/usr/bin/env python3
"""Benchmark of the B200 per-particle step: particle-steps/s on the global
forward run of 10 M particles (8 point sources, 1 kg/h each, released
continuously over 48 h; met 360x180 x 60 levels, 9 frames 3 h apart; wet
scavenging on; dt 900 s; output 360x180x5).

Set-up (untimed): the run is spun up through the C-ABI time loop
(fpg_forward_*) over its whole 48 h release window, so the timed steps see
the real population of 10 M active particles spread along the plumes.

One timed step = one 900 s sync step over all 10 M particles: met-bracket
refresh at bracket changes (every 12 steps, from a device-resident frame
ring), per-cell wet forcing at bracket changes, per-cell PBL diagnostics, a
spatial reorder by met cell every 12 steps, the fused advection +
Hanna/Langevin + dry + wet kernel, and the concentration grid at each 3-hourly
output time.  The particle state (960 MB) is larger than L2.

`e2e` runs the same steps through the driver's public calls with the met
in page-locked host memory: each met frame is copied host->device through
the driver's frame ring (fpg_forward_prefetch_frame, on a copy stream, one
bracket ahead), the bracket's precipitation goes up with its wet forcing,
and the concentration grid is read back every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

The line's "batched" object is the batched ensemble (run_batched): 256
release scenarios stepped as one population, one CUDA-graph replay per step,
against interleaved plain launches and scenario-by-scenario driver runs.
Its "adjoint" object is the source inversion's forward + backward
(run_adjoint): the 16-source, 1 M-particle inversion and the 64-instance
batched inversion with checkpoints every 8 steps.

Under torchrun each rank runs its own 10 M-particle shard (weak scaling, met
replicated, own Philox stream); the one exchange, at each output time inside
the timed region, is the NCCL sum of the ranks' integer grids.  Rank 0
prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "flexpart-gpu_b200"))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
UNIT = "particle-steps/s"
BYTES_PER_PARTICLE_STEP = 96  # read 44 B + write 52 B of SoA state, one species
ADJOINT_HBM_BUDGET = 140e9  # device bytes the batched adjoint may hold (the 150 GB budget, with margin)
# steps between spatial reorders of the population (one per simulated day at
# dt 900 s): measured at 10 M particles over 96 steps, a reorder every
# 24 / 32 / 48 / 96 steps gives 1.297 / 1.318 / 1.324 / 1.335e10
# particle-steps/s.  A reorder costs about 0.94 ms and the step kernel gains
# little from it beyond the first step after it (the turbulence mixes the
# heights within each column at once: 0.582 ms right after a reorder, 0.618
# ms from the second step on).  The default window of timed steps is one
# reorder period, and its first step reorders.
SORT_EVERY = 96
# DRAM bytes (read + write) per particle of one fused-step launch, from an
# ncu capture of a 10 M-particle launch of the global run's population
# (bench.py --quick: particles around the 8 sources, reordered by met cell
# before the timed steps): 443.2 MB read + 421.9 MB written = 86.5 B per
# particle against the algorithmic 96 B (44 B read, 52 B written); the last
# ~100 MB of writes are still in the 126 MB L2 when the kernel ends.
DRAM_BYTES_PER_PARTICLE_NCU = (443.2e6 + 421.9e6) / 10.0e6
# Warp instructions per 32 particle-steps (smsp__inst_executed.sum of the
# same capture: 553.5 M for 10 M particles).
WARP_INSTRUCTIONS_PER_32_PARTICLES_NCU = 553.5e6 / (10.0e6 / 32)


def issue_roofline(n_particles, kernel_ms, clk):
    """The fused step against the instruction-issue roofline: warp
    instructions of one launch (the ncu count per 32 particle-steps, scaled by
    the particles) over the kernel time, against 4 issues per clock on each
    SM at the SM clock sampled during the timed region."""
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    instr = WARP_INSTRUCTIONS_PER_32_PARTICLES_NCU * n_particles / 32.0
    achieved = instr / (kernel_ms / 1e3)
    peak = sms * 4 * mhz * 1e6
    return {"achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "instructions_per_launch": instr, "sm_mhz": mhz,
            "source": "smsp__inst_executed.sum of a 10M-particle ncu capture (bench.py --quick), scaled by particles"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=SORT_EVERY)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=10_000_000)
    ap.add_argument("--cpu-sample", type=int, default=200_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-scenarios", type=int, default=256)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-cbl", action="store_true", help="skip the CBL / convective-mixing kernel timings")
    ap.add_argument("--sort-every", type=int, default=SORT_EVERY,
                    help="steps between spatial reorders of the population")
    ap.add_argument("--adjoint-instances", type=int, default=64)
    ap.add_argument("--quick", action="store_true",
                    help="profiling case: no spin-up (particles scattered around the sources), no e2e, no CPU leg")
    ap.add_argument("--case", choices=["batched", "inverse"],
                    help="small profiling case, then exit: batched = 64 scenarios (~3.5 M particles) for 48 steps; "
                         "inverse = 200 k particles, 16 sources, 6 h, tape recorded in the forward")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower() in ("active", "1"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def oracle_met(scn, frames, t):
    from flexpart_gpu import synthetic
    fa, fb, _, _ = synthetic.bracket_frames(scn, t)
    return fa, fb, {"u0": frames[fa]["u"], "v0": frames[fa]["v"], "w0": frames[fa]["w"], "u1": frames[fb]["u"],
                    "v1": frames[fb]["v"], "w1": frames[fb]["w"],
                    "heights": synthetic.level_heights(scn.met.nz, scn.met.top_m)}


def oracle_steps(scn, frames, rec, threads, steps=None, seconds=None, counter0=0):
    """The oracle (C restatement of the reference step, OpenMP over
    particles) over a sample of the population: production steps with the
    same met, PBL, wet forcing and counters as the device run."""
    from flexpart_gpu import synthetic
    from flexpart_gpu.records import StepParams
    from oracle import orc

    xs, ys, zs = synthetic.velocity_scale(scn.met)
    st = orc.State.from_records(rec)
    n = len(rec)
    t = scn.end
    times = []
    k = 0
    t_start = time.perf_counter()
    while True:
        fa, fb, met = oracle_met(scn, frames, t)
        _, _, ta, tb = synthetic.bracket_frames(scn, t)
        alpha = (t - ta) / float(tb - ta)
        t0 = time.perf_counter()
        pbl = orc.pbl_diagnostics(frames[fa]["surface"], frames[fb]["surface"], alpha, scn.met.nx, scn.met.ny)
        lam, frac = orc.wet_cells(synthetic.precipitation(scn.met, fa), np.zeros(scn.met.nx * scn.met.ny),
                                  np.ones(scn.met.nx * scn.met.ny), scn.wet_a, scn.wet_b)
        prm = StepParams.production(alpha=alpha, dt_seconds=float(scn.dt), turb_dt_seconds=float(scn.dt),
                                    x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, key=scn.key,
                                    counter=(counter0 + 2 * n * k, 0, 0, 0), dry_mode=1,
                                    dry_velocity_m_s=scn.dry_velocity, wet_mode=3)
        orc.step(st, n, met, pbl, prm, wet_cells_lf=(lam, frac), wet_shape=(scn.met.nx, scn.met.ny), threads=threads)
        times.append(time.perf_counter() - t0)
        k += 1
        t += scn.dt
        el = time.perf_counter() - t_start
        if steps is not None and k >= steps:
            break
        if seconds is not None and (el >= seconds or (k >= 3 and el * (k + 1) / k > 30.0)):
            break
    return times


def legacy_steps(scn, frames, rec, threads, seconds):
    """The reference's CPU pipeline as its benchmark runs it
    (benches/advection.rs:1118-1213), restated over the oracle: the three
    wind components time-interpolated over the whole grid
    (interpolate_wind_field_linear), surface lerp + PBL diagnostics per cell,
    advection on the interpolated wind, Hanna + legacy Langevin
    (n_substeps = 0), dry and wet deposition from per-particle arrays, and
    the CPU concentration grid.  Returns the seconds of each step."""
    from flexpart_gpu import synthetic
    from flexpart_gpu.records import StepParams
    from oracle import orc

    xs, ys, zs = synthetic.velocity_scale(scn.met)
    st = orc.State.from_records(rec)
    n = len(rec)
    rng = np.random.default_rng(23)
    dry_v = rng.uniform(0.001, 0.003, n).astype(np.float32)
    wet_l = rng.uniform(0.0, 1e-3, n).astype(np.float32)
    wet_f = (np.arange(n) % 100 / 100.0).astype(np.float32)
    t = scn.end
    times = []
    t_start = time.perf_counter()
    k = 0
    while True:
        fa, fb, met = oracle_met(scn, frames, t)
        _, _, ta, tb = synthetic.bracket_frames(scn, t)
        alpha = (t - ta) / float(tb - ta)
        t0 = time.perf_counter()
        wind = {c: orc.lerp_field(met[c + "0"], met[c + "1"], alpha, threads) for c in ("u", "v", "w")}
        one = {"u0": wind["u"], "v0": wind["v"], "w0": wind["w"], "u1": wind["u"], "v1": wind["v"],
               "w1": wind["w"], "heights": met["heights"]}
        pbl = orc.pbl_diagnostics(frames[fa]["surface"], frames[fb]["surface"], alpha, scn.met.nx, scn.met.ny)
        prm = StepParams.production(alpha=0.0, dt_seconds=float(scn.dt), turb_dt_seconds=float(scn.dt),
                                    x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, key=scn.key,
                                    counter=(2 * n * k, 0, 0, 0), n_substeps=0, dry_mode=2, wet_mode=2)
        orc.step(st, n, one, pbl, prm, dry_velocity=dry_v, wet_lambda=wet_l, wet_fraction=wet_f, threads=threads)
        orc.grid(st, n, 0, 1e6, scn.outheights, scn.out_shape)
        times.append(time.perf_counter() - t0)
        k += 1
        t += scn.dt
        el = time.perf_counter() - t_start
        if el >= seconds or (k >= 3 and el * (k + 1) / k > 3 * seconds):
            break
    return times


def host_cpu():
    """CPU model name (lscpu, else /proc/cpuinfo) and whether a Rust toolchain
    is present on this host."""
    import shutil

    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                model = line.split(":", 1)[1].strip()
    except Exception:
        pass
    if model is None:
        try:
            for line in open("/proc/cpuinfo"):
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
        except Exception:
            pass
    return {"model": model, "logical_cpus": os.cpu_count(), "cargo": shutil.which("cargo")}


def cpu_figures(scn, frames, rec, threads, seconds=5.0):
    """Companion CPU numbers beside the main one: the production step on one
    core, and the reference's legacy CPU pipeline on one core and on all."""
    one = rec[:min(len(rec), 50_000)]
    t1 = oracle_steps(scn, frames, one, 1, seconds=seconds)
    out = {"production_1_core": {"value": len(one) * len(t1) / sum(t1), "unit": UNIT, "cores": 1,
                                 "sample": f"{len(one)} particles x {len(t1)} steps"}}
    for cores, sample in ((threads, rec), (1, one)):
        tl_ = legacy_steps(scn, frames, sample, cores, seconds)
        out[f"legacy_pipeline_{'1_core' if cores == 1 else 'all_cores'}"] = {
            "value": len(sample) * len(tl_) / sum(tl_), "unit": UNIT, "cores": cores,
            "sample": f"{len(sample)} particles x {len(tl_)} steps",
            "pipeline": "whole-grid wind lerp, PBL per cell, advection, Hanna + legacy Langevin (no sub-steps), "
                        "dry + wet from per-particle arrays, CPU grid (benches/advection.rs:1118-1213)"}
    out["host"] = host_cpu()
    return out


def parity_sample(ctx, scn, frames, rec, t, counter):
    """One production step of the sampled particles on the device and in the
    oracle (FP32): the largest error per field, scaled as the parity tests
    scale it (1 cell for grid positions, max(|z|, 100 m) for heights, 2 m/s
    for velocities, the mass itself)."""
    from flexpart_gpu import api, synthetic
    from flexpart_gpu.records import StepParams
    from oracle import orc

    spec = scn.met
    n = len(rec)
    fa, fb, met = oracle_met(scn, frames, t)
    _, _, ta, tb = synthetic.bracket_frames(scn, t)
    alpha = (t - ta) / float(tb - ta)
    xs, ys, zs = synthetic.velocity_scale(spec)
    prm = StepParams.production(alpha=alpha, dt_seconds=float(scn.dt), turb_dt_seconds=float(scn.dt),
                                x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, key=scn.key,
                                counter=counter, dry_mode=1, dry_velocity_m_s=scn.dry_velocity, wet_mode=3)
    precip = synthetic.precipitation(spec, fa)
    m = api.Met(ctx, spec.nx, spec.ny, spec.nz)
    m.set_level_heights(met["heights"])
    m.upload_frame(0, met["u0"], met["v0"], met["w0"])
    m.upload_frame(1, met["u1"], met["v1"], met["w1"])
    surf = api.Surface(ctx, spec.nx, spec.ny)
    surf.upload(0, frames[fa]["surface"])
    surf.upload(1, frames[fb]["surface"])
    pbl = api.Pbl(ctx, spec.nx, spec.ny)
    api.pbl_diagnostics(ctx, surf, alpha, pbl)
    wet = api.CellField(ctx, spec.nx, spec.ny)
    wet.from_precipitation(precip, None, None, scn.wet_a, scn.wet_b)
    parts = api.Particles(ctx, n)
    parts.upload(rec)
    api.step(ctx, parts, m, pbl, prm, wet_cells=wet)
    g = parts.download()
    st = orc.State.from_records(rec)
    opbl = orc.pbl_diagnostics(frames[fa]["surface"], frames[fb]["surface"], alpha, spec.nx, spec.ny)
    lam, frac = orc.wet_cells(precip, np.zeros(spec.nx * spec.ny), np.ones(spec.nx * spec.ny), scn.wet_a,
                              scn.wet_b)
    orc.step(st, n, met, opbl, prm, wet_cells_lf=(lam, frac), wet_shape=(spec.nx, spec.ny))
    o = st.to_records()
    act = (rec["flags"] & 1) != 0
    f64 = lambda a: np.asarray(a, np.float64)[act]                     # noqa: E731
    gx = lambda r, c, p: f64(r[c]) + f64(r[p])                          # noqa: E731
    zsc = np.maximum(np.maximum(np.abs(f64(o["pos_z"])), np.abs(f64(rec["pos_z"]))), 100.0)
    err = {"grid_x": np.abs(gx(g, "cell_x", "pos_x") - gx(o, "cell_x", "pos_x")),
           "grid_y": np.abs(gx(g, "cell_y", "pos_y") - gx(o, "cell_y", "pos_y")),
           "pos_z": np.abs(f64(g["pos_z"]) - f64(o["pos_z"])) / zsc}
    for f in ("turb_u", "turb_v", "turb_w", "vel_u", "vel_v", "vel_w"):
        err[f] = np.abs(f64(g[f]) - f64(o[f])) / np.maximum(np.abs(f64(o[f])), 2.0)
    mo = f64(o["mass"][:, 0])
    err["mass0"] = np.abs(f64(g["mass"][:, 0]) - mo) / np.maximum(np.abs(mo), 1e-30)
    out = {k: float(v.max()) for k, v in err.items()}
    within = {k: float((v <= 1e-5).mean()) for k, v in err.items()}
    return {"particles": int(act.sum()), "max_rel_err": out, "share_within_1e-5": within,
            "integers_bit_exact": bool(np.array_equal(g["flags"], o["flags"]) and np.array_equal(g["cbt"], o["cbt"])),
            "step": "one production step (dry + per-cell wet) of the sample, device fused_step_kernel vs FP32 oracle"}


def cpu_sample(scn, args, n):
    """A sample of particles in the plumes around the sources (no GPU)."""
    from flexpart_gpu import synthetic
    return synthetic.particles_at_sources(scn, n, seed=3)


def run_reference(args, rank, world):
    """Reference arm: the reference's CPU path is Rust and no Rust toolchain is
    present, so the oracle port of the production step is timed on the host
    cores on a sample of the same workload."""
    if rank != 0:
        return
    from flexpart_gpu import synthetic

    scn = synthetic.config1(args.particles)
    frames = synthetic.make_frames(scn.met)
    threads = os.cpu_count() or 1
    sample = min(500_000, args.particles)
    rec = cpu_sample(scn, args, sample)
    times = oracle_steps(scn, frames, rec, threads, steps=args.warmup + args.steps)[args.warmup:]
    total = sum(times)
    value = sample * len(times) / total
    extra = cpu_figures(scn, frames, rec[:200_000], threads)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": "global forward run, 10M particles from 8 sources, met 360x180x60 (CPU sample)",
                   "sample_particles": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample} plume particles per step, production step (4 sub-steps, reflection, "
                                   f"dual-time wind, dry + wet) of the oracle C restatement with {threads} OpenMP "
                                   f"threads; the reference's CPU path is Rust and no Rust toolchain is present",
                         **extra},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_batched(ctx, stream, args, rank, world):
    """The batched ensemble: 256 release scenarios (particle counts
    log-uniform in [10 k, 1 M], about 54 M in all, own source, start time and
    Philox key) on met 180x90x40 with 9 frames, 24 h at dt 900 s (97 steps),
    per-scenario output grids 180x90x3 every 3 h.  One full 24 h run is timed
    (device events, max over ranks) after a tuning pass of the launch shape;
    beside it the same run as interleaved plain launches (one fused-step
    launch per scenario per step) and as scenario-by-scenario plain driver
    runs (a subset, scaled by particle-steps)."""
    import torch
    import torch.distributed as dist

    from flexpart_gpu import api, synthetic
    from flexpart_gpu import batch as bt
    from flexpart_gpu import timeloop as tl
    import ctypes

    lib = api._lib.lib

    ens = synthetic.config2(n_scenarios=args.batch_scenarios, seed=2 + rank)
    spec = ens.met
    n = ens.n_steps
    ps = bt.particle_steps(ens)
    heights = synthetic.level_heights(spec.nz, spec.top_m)
    frames = synthetic.make_frames(spec)
    precs = [synthetic.precipitation(spec, k) for k in range(spec.n_frames)]

    def make():
        b = bt.Batch(ctx, bt.ensemble_config(ens, output_every_steps=12), bt.ensemble_scenarios(ens),
                     (spec.nx, spec.ny, spec.nz), heights, ens.outheights)
        for k, f in enumerate(frames):
            b.upload_frame(k, f, precs[k])
        return b

    def timed(fn):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ctx.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        ctx.synchronize()
        ms = a.elapsed_time(b)
        if world > 1:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        return ms

    # launch shape chosen on a copy of the run at 3/4 of its length
    b = make()
    k_tune = 3 * n // 4
    b.run(k_tune)
    best, cands = b.autotune(reps=3)
    pass_particles = bt.particle_steps(ens, k_tune, 1)
    del b
    # warm-up run, then the timed run
    b = make()
    b.tuning = best
    b.run(n)
    del b
    b = make()
    b.tuning = best
    l0 = ctx.kernel_launches
    ms = timed(lambda: b.run(n))
    launches = ctx.kernel_launches - l0
    errors = b.errors()
    del b
    b = make()
    ms_seq = timed(lambda: b.run_sequential(n))
    del b

    # end to end through the public calls: met ring from page-locked host
    # memory, run, grids back into page-locked host memory
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t, t.numpy()

    keep = []
    frames_h, precs_h = [], []
    for f, pr in zip(frames, precs):
        fh = {}
        for k in ("u", "v", "w"):
            t, fh[k] = pinned(f[k].reshape(-1))
            keep.append(t)
        t, fh["surface"] = pinned(f["surface"].view(np.uint8))
        fh["surface"] = fh["surface"].view(f["surface"].dtype)
        keep.append(t)
        t, ph = pinned(np.asarray(pr, np.float32))
        keep.append(t)
        frames_h.append(fh)
        precs_h.append(ph)
    grid_shape = (len(ens.sources),) + tuple(ens.out_shape)
    grids_h = []
    for _ in range(2):
        t, g = pinned(np.zeros(grid_shape, np.uint32))
        keep.append(t)
        grids_h.append(g)
    h2d = 0
    for f, p in zip(frames, precs):
        h2d += 3 * f["u"].nbytes + f["surface"].nbytes + p.nbytes
    b = make()
    b.tuning = best

    def e2e():
        for k, f in enumerate(frames_h):
            b.upload_frame(k, f, precs_h[k])
        b.run(n)
        b.download_grids(out=(grids_h[0], grids_h[1]))

    ms_e2e = timed(e2e)
    del b

    # scenario-by-scenario plain driver runs over a subset, every met frame
    # and precipitation field resident on the device before the timed run
    # (the driver's frame ring holds all of them; no host copy inside)
    frame_dev = [{k: api.DeviceArray.from_numpy(ctx, f[k].reshape(-1)) for k in ("u", "v", "w")}
                 | {"surface": api.DeviceArray.from_numpy(ctx, f["surface"].view(np.uint8))} for f in frames]
    precip_dev = [api.DeviceArray.from_numpy(ctx, np.ascontiguousarray(p, np.float32)) for p in precs]
    sub = min(16, len(ens.sources))
    ps_sub = 0
    t_drv = 0.0
    for s in range(sub):
        scn = ens.scenario(s)
        drv = tl.ForwardDriver(ctx, tl.scenario_config(scn), tl.scenario_releases(scn), tl.scenario_domain(scn),
                               scn.capacity, (spec.nx, spec.ny, spec.nz), heights)
        src = tl.BracketSource(scn, frames)
        cells = api.CellField(ctx, spec.nx, spec.ny)
        forcing = tl.cell_forcing(cells, dry_velocity=ens.dry_velocity)
        drv.enable_met_ring(spec.n_frames)
        for tf in range(scn.start, scn.end + spec.frame_seconds, spec.frame_seconds):
            fd_ = frame_dev[((tf - scn.start) // spec.frame_seconds) % spec.n_frames]
            drv.prefetch_frame(tf, *(fd_[k].ptr for k in ("u", "v", "w", "surface")))
        ctx.synchronize()

        def run_one():
            last = None
            for _ in range(n):
                t = drv.current_time_seconds
                fa = synthetic.bracket_frames(scn, t)[0]
                if fa != last:
                    api.check(lib.fpg_cellfield_from_precipitation(cells.h, ctypes.c_void_p(precip_dev[fa].ptr),
                                                                   None, None, ens.wet_a, ens.wet_b, None),
                              "wet cells")
                    last = fa
                drv.run_timestep(src.at(t), forcing)

        t_drv += timed(run_one) / 1e3
        one = synthetic.Ensemble(ens.name, spec, [ens.sources[s]], [ens.keys[s]], ens.start, ens.end, ens.dt,
                                 ens.out_shape, ens.outheights)
        ps_sub += bt.particle_steps(one)
        del drv, cells

    peak, peak_kind = measured_peak_hbm()
    achieved = BYTES_PER_PARTICLE_STEP * pass_particles / (best["step_ms"] / 1e3) / 1e9
    value = ps * world / (ms / 1e3)
    return {
        "workload": f"{len(ens.sources)} release scenarios, {ens.total_particles} particles (log-uniform "
                    f"[10k, 1M] per scenario), met {spec.nx}x{spec.ny}x{spec.nz}, 9 frames, 24 h, {n} steps, "
                    f"per-scenario grids {ens.out_shape[0]}x{ens.out_shape[1]}x{ens.out_shape[2]} every 3 h",
        "value": value, "unit": UNIT, "particle_steps_per_run": ps, "ms_per_run": ms,
        "gpu_launches": int(launches), "errors": errors,
        "tuning": best, "tuning_candidates": cands,
        "sequential_interleaved": {"value": ps * world / (ms_seq / 1e3), "ms_per_run": ms_seq,
                                   "path": "fpg_batch_run_sequential: one fused_step_kernel launch per scenario "
                                           "per step, shared per-step kernels, no graph"},
        "per_scenario_driver": {"value": ps_sub / t_drv, "scenarios_timed": sub, "seconds": t_drv,
                                "path": "fpg_forward_run_timestep per scenario, one plain run after another, "
                                        "every met frame resident in the driver's device frame ring"},
        "speedup": ms_seq / ms,
        "speedup_baseline": "sequential_interleaved: the same run as one plain fused-step launch per scenario "
                            "per step (per-step kernels shared)",
        "speedup_vs_interleaved": ms_seq / ms,
        "speedup_vs_per_scenario_driver": value / world / (ps_sub / t_drv),
        "e2e": {"value": ps * world / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_run": h2d,
                "d2h_bytes_per_run": 2 * grids_h[0].nbytes,
                "path": "fpg_batch_upload_frame x9 + fpg_batch_run + fpg_batch_download_grids "
                        "(page-locked host buffers)"},
        "roofline": {"bound": "hbm",
                     "kernel": "batch_step_flat_kernel" if best["particles_per_thread"] == 0 else "batch_step_kernel",
                     "particles_per_launch": pass_particles,
                     "kernel_ms": best["step_ms"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind},
    }


# ---------------------------------------------------------------------------
def run_adjoint(ctx, stream, args, rank, world):
    """Forward + adjoint of the source inversion (include/fpg_adjoint.h).

    C3: 1 M particles from 16 sources on the 90x60x20 met, 200 receptors in
    the lowest layer, 24 h; loss sum (sim - obs)^2 with obs from emissions x
    lognormal(0, 0.5) plus 10 % noise; gradient w.r.t. 16 masses, 16x3
    positions and the 90x60x20x3 wind bias.  Timed: the plain forward (no
    tape), then forward + backward with the tape recorded in the forward
    (K = 0) and with checkpoints every 8 steps (K = 8).
    C4: 64 instances (log-uniform [50 k, 2 M] particles, 8 sources and 100
    receptors each) on the 180x90x40 met, 72 h, checkpoints every 8 steps."""
    import torch
    import torch.distributed as dist

    from flexpart_gpu import batch as bt
    from flexpart_gpu import synthetic
    from flexpart_gpu.adjoint import SourceInversion, misfit, synthetic_observations

    def timed(fn):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ctx.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        ctx.synchronize()
        ms = a.elapsed_time(b)
        if world > 1:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        return ms, r

    out = {}
    inv = synthetic.config3(seed=3 + rank)
    ps = bt.particle_steps(inv.ensemble)
    res = {}
    obs = None
    for K in (8, 0):
        inv.checkpoint_every = K
        model = SourceInversion(ctx, inv)
        if obs is None:
            obs, _ = synthetic_observations(model)
        model.forward(model.mass0, model.position0)          # warm-up
        tf, sim = timed(lambda: model.forward(model.mass0, model.position0))
        loss, dsim = misfit(sim, obs)
        tb, g = timed(lambda: model.backward(dsim))
        res[K] = {"forward_ms": tf, "backward_ms": tb, "device_bytes": model.device_bytes}
        if K == 0:
            # spot check: the mass gradient of source 0 against central differences (h = 1e-3 relative)
            m0 = model.mass0.copy()
            h = 1e-3 * m0[0]
            mp, mm = m0.copy(), m0.copy()
            mp[0] += h
            mm[0] -= h
            fd = (misfit(model.forward(mp), obs)[0] - misfit(model.forward(mm), obs)[0]) / (2 * h)
            out["c3_fd_mass_source0"] = {"adjoint": float(g["mass"][0]), "fd": float(fd),
                                         "rel_err": abs(float(g["mass"][0]) - fd) / max(abs(fd), 1e-300)}
        del model
    plain = res[8]["forward_ms"]
    out["c3"] = {
        "workload": "1M particles, 16 sources, 200 receptors, met 90x60x20, 24 h (97 steps)",
        "particle_steps": ps, "plain_forward_ms": plain, "plain_forward_value": ps * world / (plain / 1e3),
        "tape_in_forward": {"forward_ms": res[0]["forward_ms"], "backward_ms": res[0]["backward_ms"],
                            "ratio_to_forward": (res[0]["forward_ms"] + res[0]["backward_ms"]) / plain,
                            "value": ps * world / ((res[0]["forward_ms"] + res[0]["backward_ms"]) / 1e3),
                            "device_bytes": res[0]["device_bytes"]},
        "checkpoint_every_8": {"forward_ms": res[8]["forward_ms"], "backward_ms": res[8]["backward_ms"],
                               "ratio_to_forward": (res[8]["forward_ms"] + res[8]["backward_ms"]) / plain,
                               "value": ps * world / ((res[8]["forward_ms"] + res[8]["backward_ms"]) / 1e3),
                               "device_bytes": res[8]["device_bytes"]},
    }
    if args.adjoint_instances > 0:
        inv4 = synthetic.config4(n_instances=args.adjoint_instances, seed=4 + rank)
        ps4 = bt.particle_steps(inv4.ensemble)
        # every window recomputed from its checkpoint: the forward is the plain
        # batched step plus the checkpoint saves, the denominator of both ratios
        model = SourceInversion(ctx, inv4)
        rng = np.random.default_rng(11)
        tf, sim = timed(lambda: model.forward(model.mass0, model.position0))
        obs4 = sim * (1.0 + 0.1 * rng.standard_normal(sim.size))
        loss, dsim = misfit(sim, obs4)
        tb, g = timed(lambda: model.backward(dsim))
        bytes0 = model.device_bytes
        del model
        # the HBM the 150 GB budget leaves holds the tape of the last W windows,
        # which the backward then reverses without recomputing them
        K = inv4.checkpoint_every
        window_bytes = K * inv4.ensemble.total_particles * 80 - inv4.ensemble.total_particles * 44
        inv4.tape_tail_windows = max(0, 1 + int((ADJOINT_HBM_BUDGET - bytes0) // window_bytes))
        model = SourceInversion(ctx, inv4)
        model.forward(model.mass0, model.position0)                           # warm-up of the taped graph
        tf_t, _ = timed(lambda: model.forward(model.mass0, model.position0))
        tb_t, _ = timed(lambda: model.backward(dsim))
        out["c4"] = {
            "workload": f"{args.adjoint_instances} inversion instances, {inv4.ensemble.total_particles} particles, "
                        f"{len(inv4.ensemble.sources)} sources, {len(inv4.receptors)} receptors, met 180x90x40, "
                        f"72 h ({inv4.ensemble.n_steps} steps), checkpoints every {K} steps",
            "particle_steps": ps4, "forward_ms": tf,
            "recompute_every_window": {"backward_ms": tb, "ratio_to_forward": (tf + tb) / tf,
                                       "device_bytes": bytes0},
            "taped_tail": {"tape_tail_windows": inv4.tape_tail_windows, "forward_ms": tf_t, "backward_ms": tb_t,
                           "ratio_to_forward": (tf_t + tb_t) / tf, "device_bytes": model.device_bytes},
        }
        # the headline is the faster mode: the recompute steps only the slots
        # whose adjoint is non-zero, so with few slots reaching receptors it
        # costs less than taping whole windows in the forward
        best_ms = min(tf + tb, tf_t + tb_t)
        out["c4"]["mode"] = "recompute_every_window" if tf + tb <= tf_t + tb_t else "taped_tail"
        out["c4"]["ratio_to_forward"] = best_ms / tf
        out["c4"]["value"] = ps4 * world / (best_ms / 1e3)
        del model
    return out


def run_cbl_convection(ctx, stream, parts, pbl, n_active, peak, args, rank, world):
    """The CBL and convective-mixing kernels over the spun-up population of
    the global run (every slot of the dispatch, n_active of them active),
    each launch timed alone with CUDA events after an L2 flush (a 256 MB
    write), 3 warm-up launches, then 10 timed.  Algorithmic bytes per slot:
    convective mixing 16 (flags + pos_z read, pos_z + cbt written; 4 for an
    inactive slot), fused CBL sampler 72 (flags, cell_x/y, pos_x/y/z read;
    the 48-byte output written), Hanna records 88 (the same 24 read, 64
    written), record-form CBL sampler 92 (flags, pos_z, 20 bytes of the
    Hanna record, 16 of uniforms read; 48 written).  Per-cell PBL gathers
    (1 MB, L2-resident) are not counted."""
    import torch

    from flexpart_gpu import cbl
    from flexpart_gpu import convection as cv
    from flexpart_gpu.records import CBL_INPUT_DTYPE, CBL_OUTPUT_DTYPE

    n = parts.dispatch_count
    flush = torch.empty(64 * 2**20, dtype=torch.int32, device="cuda")

    def per_launch_ms(fn, reps=10):
        for _ in range(3):
            fn()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            ctx.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps

    def entry(ms, bytes_):
        gbs = bytes_ / (ms / 1e3) / 1e9
        return {"ms": ms, "algorithmic_bytes": bytes_, "achieved_gbs": gbs, "frac": gbs / peak}

    out = {"slots": n, "active": n_active}
    hanna = api_device(ctx, n, cbl.HANNA_PARAMS_DTYPE)
    out_rec = api_device(ctx, n, CBL_OUTPUT_DTYPE)
    rng = np.random.default_rng(17 + rank)
    u = np.zeros(n, CBL_INPUT_DTYPE)
    u["branch_uniform"], u["gaussian_uniform0"], u["gaussian_uniform1"] = (rng.random(n, np.float32)
                                                                             for _ in range(3))
    inputs = api_device(ctx, n, CBL_INPUT_DTYPE)
    inputs.upload(u)
    del u
    ms = per_launch_ms(lambda: cbl.dispatch_hanna_params_gpu(ctx, parts, pbl, hanna))
    out["hanna_params"] = entry(ms, 88 * n_active + 68 * (n - n_active))
    ms = per_launch_ms(lambda: cbl.sample_cbl_vertical_velocity_philox(ctx, parts, pbl, (1, 2), (3, 0, 0, 0),
                                                                       out_rec))
    out["cbl_sample_philox"] = entry(ms, 72 * n_active + 52 * (n - n_active))
    ms = per_launch_ms(lambda: cbl.sample_cbl_vertical_velocity_gpu(ctx, parts, hanna, inputs, out_rec))
    out["cbl_sample_records"] = entry(ms, 92 * n_active + 52 * (n - n_active))
    del hanna, out_rec, inputs
    iface = [0.0, 400.0, 1000.0, 2000.0, 3500.0, 5000.0, 7000.0, 9000.0, 12000.0, 16000.0, 20000.0]
    _, matrix = cv.build_simplified_convection_chain(cv.SimplifiedEmanuelInputs(iface, 10.0, 2.5, 900.0), 900.0)
    mix = cv.ConvectiveMixing(ctx, matrix.level_count())
    mix.set_matrix(matrix, iface)
    ms = per_launch_ms(lambda: mix.apply(parts))
    out["convective_mixing"] = entry(ms, 16 * n_active + 4 * (n - n_active))
    out["convective_mixing"]["levels"] = matrix.level_count()
    out["l2"] = "256 MB write between timed launches"
    return out


def profile_case(name):
    """Small self-contained runs of the batched and inversion kernels for
    profilers: inputs larger than L2, a few GB on the device at most, each
    kernel launched a few dozen times."""
    from flexpart_gpu import api, synthetic

    ctx = api.Context(0)
    if name == "batched":
        from flexpart_gpu import batch as bt

        ens = synthetic.config2(n_scenarios=64, lo=10_000, hi=200_000, hours=12)
        b = bt.Batch(ctx, bt.ensemble_config(ens, output_every_steps=12), bt.ensemble_scenarios(ens),
                     (ens.met.nx, ens.met.ny, ens.met.nz), synthetic.level_heights(ens.met.nz, ens.met.top_m),
                     ens.outheights)
        bt.upload_ensemble_met(b, ens)
        b.run(ens.n_steps)
        ctx.synchronize()
        print("batched", ens.total_particles, "particles", ens.n_steps, "steps, errors", b.errors())
    else:
        from flexpart_gpu.adjoint import SourceInversion, misfit

        inv = synthetic.config3(n_particles=200_000, hours=6)
        inv.checkpoint_every = 0
        model = SourceInversion(ctx, inv)
        sim = model.forward(model.mass0, model.position0)
        loss, d = misfit(sim, sim * 1.1 + 1e-12)
        g = model.backward(d)
        print("inverse loss", loss, "grad mass norm", float(np.linalg.norm(g["mass"])))


def api_device(ctx, n, dtype):
    from flexpart_gpu import api
    return api.DeviceArray(ctx, n, dtype)


# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.case:
        profile_case(args.case)
        return

    import ctypes

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120))

    from flexpart_gpu import api, synthetic
    from flexpart_gpu import distributed as fd
    from flexpart_gpu import timeloop as tl
    from flexpart_gpu.records import StepParams

    lib = api._lib.lib
    scn = synthetic.config1(args.particles)
    spec = scn.met
    frames = synthetic.make_frames(spec)
    heights = synthetic.level_heights(spec.nz, spec.top_m)
    xs, ys, zs = synthetic.velocity_scale(spec)
    release_end = scn.end
    scn.end = release_end + (2 * (args.warmup + args.steps) + 8) * scn.dt   # room for the timed steps
    precip = [synthetic.precipitation(spec, k) for k in range(spec.n_frames)]

    ctx = api.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)

    # ---- spin-up through the C-ABI time loop: 48 h of release ----
    t_spin = time.perf_counter()
    cfg = tl.scenario_config(scn, sort_interval_steps=args.sort_every,
                             initial_philox_counter=fd.rank_counter((0, 0, 0, 0), rank))
    drv = tl.ForwardDriver(ctx, cfg, tl.scenario_releases(scn), tl.scenario_domain(scn), args.particles,
                           (spec.nx, spec.ny, spec.nz), heights)
    src = tl.BracketSource(scn, frames)
    wet_spin = api.CellField(ctx, spec.nx, spec.ny)
    wet_spin.from_precipitation(precip[0], None, None, scn.wet_a, scn.wet_b)
    forcing = tl.cell_forcing(wet_spin, dry_velocity=scn.dry_velocity)
    if args.quick:
        args.no_e2e = args.no_cpu_baseline = True
        parts = api.Particles(ctx, args.particles)
        parts.upload(synthetic.particles_at_sources(scn, args.particles, seed=3 + rank))
        n_active, counter = args.particles, [0, 0, 0, 0]
    else:
        rep = None
        while drv.current_time_seconds <= release_end:
            rep = drv.run_timestep(src.at(drv.current_time_seconds), forcing)
        drv.finalize()
        parts = drv.particles
        n_active = int(rep.active_particle_count)
        counter = list(rep.next_philox_counter)
    spin_s = time.perf_counter() - t_spin

    # ---- device-resident met ring for the timed loop ----
    frame_dev = [tuple(api.DeviceArray.from_numpy(ctx, f[k].reshape(-1)) for k in ("u", "v", "w")) for f in frames]
    # the surface frames and precipitation fields too: every input of the
    # timed loop is resident in HBM before it starts
    surf_dev = [api.DeviceArray.from_numpy(ctx, f["surface"].view(np.uint8)) for f in frames]
    precip_dev = [api.DeviceArray.from_numpy(ctx, np.ascontiguousarray(p, np.float32).reshape(-1)) for p in precip]
    met = api.Met(ctx, spec.nx, spec.ny, spec.nz)
    met.set_level_heights(heights)
    surf = api.Surface(ctx, spec.nx, spec.ny)
    pbl = api.Pbl(ctx, spec.nx, spec.ny)
    wet = api.CellField(ctx, spec.nx, spec.ny)
    grid = api.Grid(ctx, *scn.out_shape)
    sorter = api.Sorter(ctx, args.particles)
    state = {"bracket": None, "counter": counter, "t": drv.current_time_seconds, "k": 0}

    def set_bracket(fa, fb):
        (u0, v0, w0), (u1, v1, w1) = frame_dev[fa], frame_dev[fb]
        api.check(lib.fpg_met_upload_bracket_device(met.h, *(ctypes.c_void_p(x.ptr) for x in (u0, v0, w0, u1, v1, w1)),
                                                    None), "met bracket")
        for which, fi in ((0, fa), (1, fb)):
            api.check(lib.fpg_surface_upload(surf.h, which, ctypes.c_void_p(surf_dev[fi].ptr), None), "surface")
        api.check(lib.fpg_cellfield_from_precipitation(wet.h, ctypes.c_void_p(precip_dev[fa].ptr), None, None,
                                                       scn.wet_a, scn.wet_b, None), "wet cells")

    ev = []
    n_out_cells = scn.out_shape[0] * scn.out_shape[1] * scn.out_shape[2]
    # torch's collectives run on its current stream: make that the library's stream
    torch.cuda.set_stream(stream)

    stage_ev = {"bracket": [], "reorder": [], "pbl": [], "grid": []}

    def staged(name, record, fn):
        if not record:
            return fn()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        stage_ev[name].append((a, b))
        return r

    def one_step(record: bool):
        t = state["t"]
        fa, fb, ta, tb = synthetic.bracket_frames(scn, t)
        if state["bracket"] != (fa, fb, ta):
            staged("bracket", record, lambda: set_bracket(fa, fb))
            state["bracket"] = (fa, fb, ta)
        alpha = (t - ta) / float(tb - ta)
        # the first timed step reorders, then every sort_every steps: any window
        # of timed steps pays for at least one reorder
        if (state["k"] - args.warmup) % args.sort_every == 0:
            staged("reorder", record, lambda: sorter.sort(parts, met))
        staged("pbl", record, lambda: api.pbl_diagnostics(ctx, surf, alpha, pbl))
        prm = StepParams.production(alpha=alpha, dt_seconds=float(scn.dt), turb_dt_seconds=float(scn.dt),
                                    x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, key=scn.key,
                                    counter=state["counter"], dry_mode=1, dry_velocity_m_s=scn.dry_velocity,
                                    wet_mode=3)
        if record:
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
        state["counter"] = api.step(ctx, parts, met, pbl, prm, wet_cells=wet)
        if record:
            b.record(stream)
            ev.append((a, b))
        if state["k"] % 12 == 11:
            staged("grid", record, lambda: grid.accumulate(parts, 0, 1e6, scn.outheights))
            if world > 1:
                # the one exchange: the ranks' integer grids summed (mod 2^32) over NCCL
                fd.allreduce_grids_device(lib.fpg_grid_counts_device(grid.h), lib.fpg_grid_mass_device(grid.h),
                                          n_out_cells)
        state["t"] = t + scn.dt
        state["k"] += 1

    # launch shape of the step kernel: every compiled shape timed on the
    # spun-up population from one snapshot (restored), the fastest kept
    t0_ = state["t"]
    fa_, fb_, ta_, tb_ = synthetic.bracket_frames(scn, t0_)
    set_bracket(fa_, fb_)
    state["bracket"] = (fa_, fb_, ta_)
    alpha_ = (t0_ - ta_) / float(tb_ - ta_)
    api.pbl_diagnostics(ctx, surf, alpha_, pbl)
    tune_prm = StepParams.production(alpha=alpha_, dt_seconds=float(scn.dt), turb_dt_seconds=float(scn.dt),
                                     x_grid_per_meter=xs, y_grid_per_meter=ys, z_grid_per_meter=zs, key=scn.key,
                                     counter=state["counter"], dry_mode=1, dry_velocity_m_s=scn.dry_velocity,
                                     wet_mode=3)
    sorter.sort(parts, met)
    step_best, step_cands = api.step_autotune(ctx, parts, met, pbl, tune_prm, wet_cells=wet, reps=3)
    ctx.synchronize()

    for _ in range(args.warmup):
        one_step(False)
    ctx.synchronize()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    start_ev = torch.cuda.Event(enable_timing=True)
    end_ev = torch.cuda.Event(enable_timing=True)
    launches0 = ctx.kernel_launches
    start_ev.record(stream)
    for _ in range(args.steps):
        one_step(True)
    end_ev.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    launches = ctx.kernel_launches - launches0
    clk = clocks.stop()
    elapsed_ms = start_ev.elapsed_time(end_ev)
    if world > 1:
        tt = torch.tensor([elapsed_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed_ms = float(tt.item())
    kernel_ms = [a.elapsed_time(b) for a, b in ev]
    avg_kernel_ms = sum(kernel_ms) / len(kernel_ms)
    stages = {"step_kernel_ms": avg_kernel_ms}
    for name, evs in stage_ev.items():
        if evs:
            stages[f"{name}_ms"] = sum(a.elapsed_time(b) for a, b in evs) / len(evs)
            stages[f"{name}_per_window"] = len(evs)
    value = n_active * args.steps * world / (elapsed_ms / 1e3)
    peak, peak_kind = measured_peak_hbm()
    achieved = BYTES_PER_PARTICLE_STEP * n_active / (avg_kernel_ms / 1e3) / 1e9

    # ---- end to end through the driver's public call, met from the host ----
    e2e = None
    if not args.no_e2e:
        ncell = scn.out_shape[0] * scn.out_shape[1] * scn.out_shape[2]
        counts_h = torch.empty(ncell, dtype=torch.int32, pin_memory=True)
        mass_h = torch.empty(ncell, dtype=torch.int32, pin_memory=True)
        h2d = {"bytes": 0}
        seen = {"bracket": None, "prefetched": set()}
        oh = np.asarray(scn.outheights, np.float32)
        # the met frames in page-locked host memory (the run's inputs), streamed
        # to the device through the driver's frame ring one bracket ahead
        pinned = []
        for f in frames:
            pf = {}
            for k in ("u", "v", "w"):
                pf[k] = torch.from_numpy(np.ascontiguousarray(f[k].reshape(-1))).pin_memory()
            pf["surface"] = torch.from_numpy(f["surface"].view(np.uint8)).pin_memory()
            pinned.append(pf)
        precip_pinned = [torch.from_numpy(np.ascontiguousarray(p_, np.float32).reshape(-1)).pin_memory()
                         for p_ in precip]
        drv.enable_met_ring(3)
        fs = spec.frame_seconds
        copy_stream = torch.cuda.Stream()

        def prefetch(tf):
            if tf in seen["prefetched"]:
                return
            pf = pinned[((tf - scn.start) // fs) % spec.n_frames]
            drv.prefetch_frame(tf, *(pf[k].data_ptr() for k in ("u", "v", "w", "surface")))
            seen["prefetched"].add(tf)
            h2d["bytes"] += sum(pf[k].numel() * pf[k].element_size() for k in pf)

        def e2e_step():
            t = drv.current_time_seconds
            fa, fb, ta, tb = synthetic.bracket_frames(scn, t)
            prefetch(ta)
            prefetch(tb)
            if seen["bracket"] != (fa, fb, ta):
                # the precipitation field of the bracket goes up with its wet forcing
                wet_spin.from_precipitation(precip_pinned[fa].numpy(), None, None, scn.wet_a, scn.wet_b, sync=False)
                h2d["bytes"] += precip[fa].nbytes
                seen["bracket"] = (fa, fb, ta)
            drv.run_timestep(src.at(t), forcing)
            prefetch(tb + fs)       # the next bracket's new frame, while this one is in use
            api.check(lib.fpg_forward_accumulate_grid(drv.h, grid.h, 0, 1e6, ctypes.c_void_p(oh.ctypes.data),
                                                      oh.size), "grid")
            # the step's grid to pinned host memory on the copy stream, under the next step's compute
            grid.download_async(counts_h.data_ptr(), mass_h.data_ptr(), ctypes.c_void_p(copy_stream.cuda_stream))

        for _ in range(args.warmup):
            e2e_step()
        h2d["bytes"] = 0
        seen["bracket"] = None
        ring0 = drv.met_ring_stats()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ctx.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            e2e_step()
        stream.wait_stream(copy_stream)            # the last grid is on the host inside the timed region
        b.record(stream)
        ctx.synchronize()
        ms = a.elapsed_time(b)
        if world > 1:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        e2e = {"value": n_active * args.steps * world / (ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": h2d["bytes"] // args.steps, "d2h_bytes_per_step": 2 * ncell * 4,
               "ms_per_step": ms / args.steps,
               "met_ring": dict(zip(("bracket_hits", "host_uploads"),
                                    (a1 - a0 for a1, a0 in zip(drv.met_ring_stats(), ring0)))),
               "path": "fpg_forward_prefetch_frame (met frames from pinned host memory, one bracket ahead) + "
                       "fpg_forward_run_timestep + fpg_forward_accumulate_grid + fpg_grid_download_async "
                       "(every step's grid to pinned host memory on a copy stream)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = min(args.cpu_sample, n_active)
        rec = parts.download(0, sample)
        times = oracle_steps(scn, frames, rec, threads, seconds=10.0)
        cpu = {"value": sample * len(times) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"the first {sample} particles of the spun-up population x {len(times)} production steps "
                         f"(oracle C restatement, {threads} OpenMP threads, {sum(times):.1f} s)",
               "parity": parity_sample(ctx, scn, frames, rec, scn.end, [0, 0, 0, 0]),
               **cpu_figures(scn, frames, rec, threads)}

    batched = None
    if not args.no_batched and not args.quick:
        batched = run_batched(ctx, stream, args, rank, world)
    adjoint = None
    if not args.no_adjoint and not args.quick:
        adjoint = run_adjoint(ctx, stream, args, rank, world)
    cbl_conv = None
    if not args.no_cbl:
        cbl_conv = run_cbl_convection(ctx, stream, parts, pbl, n_active, peak, args, rank, world)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "global forward run: 10M particles from 8 sources released over 48 h "
                                   "(spun up), met 360x180x60, 9 frames 3 h apart, wet scavenging on, dt 900 s, "
                                   "output 360x180x5 every 3 h",
                       "particles_per_gpu": n_active, "met": [spec.nx, spec.ny, spec.nz],
                       "sort_every_steps": args.sort_every, "spin_up_s": round(spin_s, 1),
                       "l2": "inputs larger than L2 (960 MB particle state per step)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": DRAM_BYTES_PER_PARTICLE_NCU * n_active,
                         "traffic_source": "ncu dram__bytes_read+write of a 10M-particle launch (bench.py --quick), "
                                           "scaled by particles",
                         "peak_kind": peak_kind,
                         "kernel": "fused_step_kernel", "kernel_ms": avg_kernel_ms,
                         "bytes_per_launch": BYTES_PER_PARTICLE_STEP * n_active,
                         # the bound that binds: warp-instruction issue (148 SMs x 4 per clock)
                         "issue": issue_roofline(n_active, avg_kernel_ms, clk)},
            "stages": stages,
            "step_tuning": {"best": step_best, "candidates": step_cands,
                            "how": "fpg_step_autotune on the spun-up, reordered population: each compiled shape "
                                   "timed (best of 3) from one restored snapshot"},
            "clocks": clk,
            "gpu_launches": int(launches),
            "e2e": e2e,
            "cpu_baseline": cpu,
            "batched": batched,
            "adjoint": adjoint,
            "cbl_convection": cbl_conv,
        }
        print(json.dumps(line), flush=True)
    del drv
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
