"""Small, self-contained runs of the batched and inversion kernels for
profilers (inputs larger than L2, a few GB on the device at most, each
kernel launched a few dozen times).

    python -m flexpart_gpu.profile_cases batched    # batch_step_kernel: 64 scenarios, ~4 M particles, 48 steps
    python -m flexpart_gpu.profile_cases inverse    # inverse_tape_kernel / inverse_adjoint_kernel:
                                                    # 200 k particles, 16 sources, 6 h, tape in the forward
"""
from __future__ import annotations

import sys

import numpy as np


def batched():
    from . import api, synthetic
    from . import batch as bt

    ctx = api.Context(0)
    ens = synthetic.config2(n_scenarios=64, lo=10_000, hi=200_000, hours=12)
    b = bt.Batch(ctx, bt.ensemble_config(ens, output_every_steps=12), bt.ensemble_scenarios(ens),
                 (ens.met.nx, ens.met.ny, ens.met.nz), synthetic.level_heights(ens.met.nz, ens.met.top_m),
                 ens.outheights)
    bt.upload_ensemble_met(b, ens)
    b.run(ens.n_steps)
    ctx.synchronize()
    print("batched", ens.total_particles, "particles", ens.n_steps, "steps, errors", b.errors())


def inverse():
    from . import api, synthetic
    from .adjoint import SourceInversion, misfit

    ctx = api.Context(0)
    inv = synthetic.config3(n_particles=200_000, hours=6)
    inv.checkpoint_every = 0
    model = SourceInversion(ctx, inv)
    sim = model.forward(model.mass0, model.position0)
    loss, d = misfit(sim, sim * 1.1 + 1e-12)
    g = model.backward(d)
    print("inverse loss", loss, "grad mass norm", float(np.linalg.norm(g["mass"])))


if __name__ == "__main__":
    {"batched": batched, "inverse": inverse}[sys.argv[1] if len(sys.argv) > 1 else "batched"]()
