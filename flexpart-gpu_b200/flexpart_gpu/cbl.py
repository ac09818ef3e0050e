"""Convective-boundary-layer turbulence on the device: per-slot Hanna
parameters and the CBL skewed vertical-velocity sampler.

Mirrors the reference's GPU entry points:

* ``dispatch_hanna_params_gpu`` / ``compute_hanna_params_gpu``
  (src/gpu/hanna.rs:212-330): one HannaParams record per slot from the PBL
  fields at the particle's cell;
* ``update_particles_turbulence_langevin_gpu`` (src/gpu/langevin.rs:
  248-329): the Langevin update from those records (the reference's
  validation and backward path; the fused step computes the same);
* ``sample_cbl_vertical_velocity_gpu`` (src/gpu/cbl.rs:189-319): the
  bi-Gaussian PDF of w' and one sample per slot from caller uniforms;
* ``sample_cbl_vertical_velocity_philox``: the same sample with sigma_w
  formed at the slot's cell and the uniforms drawn from Philox on the
  device (the reference's sample_cbl_vertical_velocity_with_rng,
  physics/cbl.rs:291-295, one stream per slot starting at counter + slot).

Like the reference's dispatch, the sampler does not write the particles'
turbulence memory (src/gpu/cbl.rs:13-16).  Errors raise FpgError with the
reference's error kinds (MismatchedInputLengths -> LENGTH_MISMATCH,
ZeroPblShape -> ZERO_SHAPE).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .api import Context, DeviceArray, Particles, Pbl, _u32arr, _vp
from .records import CBL_INPUT_DTYPE, CBL_OUTPUT_DTYPE, HANNA_PARAMS_DTYPE

__all__ = [
    "HANNA_PARAMS_DTYPE", "CBL_INPUT_DTYPE", "CBL_OUTPUT_DTYPE", "sampling_inputs",
    "dispatch_hanna_params_gpu", "compute_hanna_params_gpu", "update_particles_turbulence_langevin_gpu",
    "sample_cbl_vertical_velocity_gpu",
    "sample_cbl_vertical_velocity_philox",
]


def sampling_inputs(branch_uniform, gaussian_uniform0, gaussian_uniform1) -> np.ndarray:
    """CblSamplingInput records (CblSamplingInput::new, src/gpu/cbl.rs:52-61)."""
    b = np.atleast_1d(np.asarray(branch_uniform, np.float32))
    out = np.zeros(b.size, CBL_INPUT_DTYPE)
    out["branch_uniform"] = b
    out["gaussian_uniform0"] = gaussian_uniform0
    out["gaussian_uniform1"] = gaussian_uniform1
    return out


def dispatch_hanna_params_gpu(ctx: Context, particles: Particles, pbl: Pbl, output: DeviceArray | None = None,
                              stream=None) -> DeviceArray:
    """Fills `output` (a device array of HANNA_PARAMS_DTYPE, one record per
    slot of the dispatch count; allocated when not given) and returns it."""
    n = particles.dispatch_count
    if output is None:
        output = DeviceArray(ctx, n, HANNA_PARAMS_DTYPE)
    check(lib.fpg_dispatch_hanna_params(ctx.h, particles.h, pbl.h, _vp(output.ptr), output.n, stream),
          "fpg_dispatch_hanna_params")
    return output


def compute_hanna_params_gpu(ctx: Context, particles: Particles, pbl: Pbl) -> np.ndarray:
    """Per-slot HannaParams downloaded to the host (zeros for inactive slots)."""
    if particles.dispatch_count == 0:
        return np.zeros(0, HANNA_PARAMS_DTYPE)
    return dispatch_hanna_params_gpu(ctx, particles, pbl).numpy()


def update_particles_turbulence_langevin_gpu(ctx: Context, particles: Particles, hanna_params, dt: float,
                                             rho_grad_over_rho: float, n_substeps: int, min_height_m: float, key,
                                             counter, stream=None):
    """The Langevin update from per-slot HannaParams records (a host record
    array or a DeviceArray of HANNA_PARAMS_DTYPE): the reference's separated
    Hanna -> Langevin path (src/gpu/langevin.rs:248-329).  Returns the next
    Philox counter."""
    h_dev, n_h = _device(ctx, hanna_params, HANNA_PARAMS_DTYPE)
    nxt = (ctypes.c_uint32 * 4)()
    check(lib.fpg_langevin_with_hanna(ctx.h, particles.h, _vp(h_dev.ptr), n_h, dt, rho_grad_over_rho, n_substeps,
                                      min_height_m, _u32arr(key, 2), _u32arr(counter, 4), nxt, stream),
          "fpg_langevin_with_hanna")
    return list(nxt)


def _device(ctx, a, dtype):
    if isinstance(a, DeviceArray):
        return a, a.n
    a = np.ascontiguousarray(a, dtype)
    return DeviceArray.from_numpy(ctx, a), a.size


def sample_cbl_vertical_velocity_gpu(ctx: Context, particles: Particles, hanna_params, inputs,
                                     output: DeviceArray | None = None, stream=None):
    """One CblSamplingOutput per slot.  `hanna_params` and `inputs` are host
    record arrays or DeviceArrays; with host inputs and no `output` the
    result comes back as a host array, otherwise `output` is filled and
    returned."""
    n = particles.dispatch_count
    h_dev, n_h = _device(ctx, hanna_params, HANNA_PARAMS_DTYPE)
    i_dev, n_i = _device(ctx, inputs, CBL_INPUT_DTYPE)
    download = output is None
    out = output if output is not None else DeviceArray(ctx, n, CBL_OUTPUT_DTYPE)
    check(lib.fpg_cbl_sample(ctx.h, particles.h, _vp(h_dev.ptr), n_h, _vp(i_dev.ptr), n_i, _vp(out.ptr), stream),
          "fpg_cbl_sample")
    if not download:
        return out
    return out.numpy()[:n] if n else np.zeros(0, CBL_OUTPUT_DTYPE)


def sample_cbl_vertical_velocity_philox(ctx: Context, particles: Particles, pbl: Pbl, key, counter,
                                        output: DeviceArray | None = None, stream=None):
    """The fused sampler: sigma_w at the slot's PBL cell and the uniforms of
    Philox block counter + slot under `key` (two u32) — no per-slot inputs in
    memory.  Returns a host array unless `output` is given."""
    n = particles.dispatch_count
    download = output is None
    out = output if output is not None else DeviceArray(ctx, n, CBL_OUTPUT_DTYPE)
    check(lib.fpg_cbl_sample_philox(ctx.h, particles.h, pbl.h, _u32arr(key, 2), _u32arr(counter, 4), _vp(out.ptr),
                                    stream), "fpg_cbl_sample_philox")
    if not download:
        return out
    return out.numpy()[:n] if n else np.zeros(0, CBL_OUTPUT_DTYPE)
