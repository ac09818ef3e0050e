"""Host-side handles over the C ABI (include/fpg.h).

Each class owns one C handle and mirrors the reference object it replaces:
`Particles` is ParticleBuffers (src/gpu/buffers.rs:377-510), `Met` is
DualWindBuffers (buffers.rs:801-950), `Pbl` is PblBuffers (buffers.rs:955-1060),
`Surface` is SurfaceFieldBuffer (src/gpu/pbl.rs:142-240), `Grid` is
ConcentrationGridIoBuffers (src/gpu/gridding.rs:126-220) and `Compaction`
is CompactionBuffers (src/gpu/compaction.rs).  Errors raise FpgError carrying
the C status (the reference's error enums, include/fpg.h).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib
from .records import (
    FIELD_DTYPE,
    FIELD_ID,
    PARTICLE_DTYPE,
    SURFACE_DTYPE,
    PblOptions,
    StepParams,
)

_vp = ctypes.c_void_p


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def _u32arr(vals, n):
    return (ctypes.c_uint32 * n)(*[int(v) & 0xFFFFFFFF for v in vals])


class Context:
    def __init__(self, device: int = 0):
        h = _vp()
        check(lib.fpg_ctx_create(device, ctypes.byref(h)), "fpg_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            lib.fpg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib.fpg_ctx_synchronize(self.h, None), "fpg_ctx_synchronize")

    @property
    def kernel_launches(self) -> int:
        return int(lib.fpg_ctx_kernel_launches(self.h))

    @property
    def stream(self):
        return lib.fpg_ctx_stream(self.h)


class DeviceArray:
    """A plain device buffer (fpg_device_alloc)."""

    def __init__(self, ctx: Context, n: int, dtype=np.float32):
        self.ctx, self.n, self.dtype = ctx, n, np.dtype(dtype)
        h = _vp()
        check(lib.fpg_device_alloc(ctx.h, max(n, 1) * self.dtype.itemsize, ctypes.byref(h)), "fpg_device_alloc")
        self.ptr = h.value

    @classmethod
    def from_numpy(cls, ctx: Context, a: np.ndarray) -> "DeviceArray":
        a = np.ascontiguousarray(a)
        d = cls(ctx, a.size, a.dtype)
        d.upload(a)
        return d

    def upload(self, a: np.ndarray):
        a = np.ascontiguousarray(a, self.dtype)
        check(lib.fpg_memcpy(self.ctx.h, _vp(self.ptr), _p(a), a.nbytes, 0, None), "fpg_memcpy")
        self.ctx.synchronize()

    def zero(self):
        check(lib.fpg_memset(self.ctx.h, _vp(self.ptr), 0, self.n * self.dtype.itemsize, None), "fpg_memset")

    def numpy(self) -> np.ndarray:
        out = np.empty(self.n, self.dtype)
        check(lib.fpg_memcpy(self.ctx.h, _p(out), _vp(self.ptr), out.nbytes, 1, None), "fpg_memcpy")
        return out

    def free(self):
        # handles die before their context (include/fpg.h); a buffer collected
        # after its context closed is left to the process exit
        if self.ptr and self.ctx.h:
            lib.fpg_device_free(self.ctx.h, _vp(self.ptr))
        self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Particles:
    def __init__(self, ctx: Context, capacity: int):
        self.ctx = ctx
        h = _vp()
        check(lib.fpg_particles_create(ctx.h, capacity, ctypes.byref(h)), "fpg_particles_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_particles_destroy(self.h)
        except Exception:
            pass

    @property
    def capacity(self) -> int:
        return int(lib.fpg_particles_capacity(self.h))

    @property
    def dispatch_count(self) -> int:
        return int(lib.fpg_particles_dispatch_count(self.h))

    @dispatch_count.setter
    def dispatch_count(self, n: int):
        check(lib.fpg_particles_set_dispatch_count(self.h, n), "fpg_particles_set_dispatch_count")

    def upload(self, records: np.ndarray, first: int = 0):
        rec = np.ascontiguousarray(records, PARTICLE_DTYPE)
        check(lib.fpg_particles_upload(self.h, first, len(rec), _p(rec), None), "fpg_particles_upload")

    def upload_slots(self, slots, records: np.ndarray):
        rec = np.ascontiguousarray(records, PARTICLE_DTYPE)
        sl = np.ascontiguousarray(slots, np.uint32)
        check(lib.fpg_particles_upload_slots(self.h, _p(sl), len(sl), _p(rec), None), "fpg_particles_upload_slots")

    def download(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.capacity - first if count is None else count
        out = np.zeros(count, PARTICLE_DTYPE)
        check(lib.fpg_particles_download(self.h, first, count, _p(out), None), "fpg_particles_download")
        return out

    def field_ptr(self, name: str) -> int:
        return lib.fpg_particles_field(self.h, FIELD_ID[name])

    def write_field(self, name: str, host: np.ndarray, first: int = 0):
        a = np.ascontiguousarray(host, FIELD_DTYPE[name])
        check(lib.fpg_particles_copy_field(self.h, FIELD_ID[name], first, a.size, _p(a), 1, None),
              "fpg_particles_copy_field")
        self.ctx.synchronize()

    def read_field(self, name: str, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.capacity - first if count is None else count
        out = np.empty(count, FIELD_DTYPE[name])
        check(lib.fpg_particles_copy_field(self.h, FIELD_ID[name], first, count, _p(out), 0, None),
              "fpg_particles_copy_field")
        return out


class Met:
    def __init__(self, ctx: Context, nx: int, ny: int, nz: int):
        self.ctx, self.shape = ctx, (nx, ny, nz)
        h = _vp()
        check(lib.fpg_met_create(ctx.h, nx, ny, nz, ctypes.byref(h)), "fpg_met_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_met_destroy(self.h)
        except Exception:
            pass

    def upload_frame(self, which: int, u, v, w):
        arrs = [np.ascontiguousarray(x, np.float32).reshape(-1) for x in (u, v, w)]
        for a in arrs:
            if a.size != self.shape[0] * self.shape[1] * self.shape[2]:
                raise ValueError("wind frame size does not match the met shape")
        check(lib.fpg_met_upload_frame(self.h, which, *[_p(a) for a in arrs], None), "fpg_met_upload_frame")
        self.ctx.synchronize()

    def upload_bracket_device(self, frame0, frame1, stream=None):
        """Both frames from device arrays ((u, v, w) DeviceArrays each) in one
        pass (fpg_met_upload_bracket_device)."""
        n = self.shape[0] * self.shape[1] * self.shape[2]
        ptrs = []
        for a in (*frame0, *frame1):
            if a.n != n:
                raise ValueError("wind frame size does not match the met shape")
            ptrs.append(ctypes.c_void_p(a.ptr))
        check(lib.fpg_met_upload_bracket_device(self.h, *ptrs, stream), "fpg_met_upload_bracket_device")

    def set_level_heights(self, heights):
        h = np.ascontiguousarray(heights, np.float32)
        check(lib.fpg_met_set_level_heights(self.h, _p(h), h.size), "fpg_met_set_level_heights")


PBL_FIELDS = ("ustar", "wstar", "hmix", "oli", "sshf", "ssr", "surfstr")


class Pbl:
    def __init__(self, ctx: Context, nx: int, ny: int):
        self.ctx, self.shape = ctx, (nx, ny)
        h = _vp()
        check(lib.fpg_pbl_create(ctx.h, nx, ny, ctypes.byref(h)), "fpg_pbl_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_pbl_destroy(self.h)
        except Exception:
            pass

    def upload(self, ustar, wstar, hmix, oli, sshf=None, ssr=None, surfstr=None):
        n = self.shape[0] * self.shape[1]
        arrs = []
        for a in (ustar, wstar, hmix, oli, sshf, ssr, surfstr):
            arrs.append(None if a is None else np.ascontiguousarray(a, np.float32).reshape(n))
        check(lib.fpg_pbl_upload(self.h, *[None if a is None else _p(a) for a in arrs], None), "fpg_pbl_upload")
        self.ctx.synchronize()

    def download(self) -> dict:
        n = self.shape[0] * self.shape[1]
        out = {k: np.empty(n, np.float32) for k in PBL_FIELDS}
        check(lib.fpg_pbl_download(self.h, *[_p(out[k]) for k in PBL_FIELDS], None), "fpg_pbl_download")
        return out


class Surface:
    def __init__(self, ctx: Context, nx: int, ny: int):
        self.ctx, self.shape = ctx, (nx, ny)
        h = _vp()
        check(lib.fpg_surface_create(ctx.h, nx, ny, ctypes.byref(h)), "fpg_surface_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_surface_destroy(self.h)
        except Exception:
            pass

    def upload(self, which: int, cells: np.ndarray):
        c = np.ascontiguousarray(cells, SURFACE_DTYPE)
        if c.size != self.shape[0] * self.shape[1]:
            raise ValueError("surface cell count does not match the shape")
        check(lib.fpg_surface_upload(self.h, which, _p(c), None), "fpg_surface_upload")
        self.ctx.synchronize()


def pbl_diagnostics(ctx: Context, surface: Surface, alpha: float, pbl: Pbl, options: PblOptions | None = None):
    opts = options or PblOptions.default()
    check(lib.fpg_pbl_diagnostics(ctx.h, surface.h, alpha, ctypes.byref(opts), pbl.h, None), "fpg_pbl_diagnostics")


class CellField:
    def __init__(self, ctx: Context, nx: int, ny: int):
        self.ctx, self.shape = ctx, (nx, ny)
        h = _vp()
        check(lib.fpg_cellfield_create(ctx.h, nx, ny, ctypes.byref(h)), "fpg_cellfield_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_cellfield_destroy(self.h)
        except Exception:
            pass

    def upload(self, lam, frac):
        l_ = np.ascontiguousarray(lam, np.float32).reshape(-1)
        f_ = np.ascontiguousarray(frac, np.float32).reshape(-1)
        check(lib.fpg_cellfield_upload(self.h, _p(l_), _p(f_), None), "fpg_cellfield_upload")
        self.ctx.synchronize()

    def from_precipitation(self, lsp, convp=None, cloud_cover=None, a: float = 1.0e-4, b: float = 0.8,
                           sync: bool = True):
        """Per-cell wet forcing from host precipitation fields.  With
        sync=False the call returns once the work is queued: the arrays must
        then stay alive and unchanged until the stream has run it (page-locked
        arrays are copied asynchronously)."""
        arrs = [None if x is None else np.ascontiguousarray(x, np.float32).reshape(-1) for x in (lsp, convp, cloud_cover)]
        check(lib.fpg_cellfield_from_precipitation(self.h, *[None if x is None else _p(x) for x in arrs], a, b, None),
              "fpg_cellfield_from_precipitation")
        if sync:
            self.ctx.synchronize()


def step(ctx: Context, particles: Particles, met: Met | None, pbl: Pbl | None, params: StepParams,
         wet_cells: CellField | None = None, stream=None):
    """fpg_step: one fused pass; returns the next Philox counter."""
    if wet_cells is not None:
        params.wet_cells = wet_cells.h.value
    nxt = (ctypes.c_uint32 * 4)()
    check(lib.fpg_step(ctx.h, particles.h, met.h if met else None, pbl.h if pbl else None,
                       ctypes.byref(params), nxt, stream), "fpg_step")
    return list(nxt)


def step_tuning_candidates() -> list[dict]:
    """The compiled launch shapes of fpg_step."""
    from .records import BatchTuning

    n = lib.fpg_step_tuning_candidates(None, 0)
    res = (BatchTuning * n)()
    lib.fpg_step_tuning_candidates(res, n)
    return [r.as_dict() for r in res]


def step_autotune(ctx: Context, particles: Particles, met: Met | None, pbl: Pbl | None, params: StepParams,
                  wet_cells: CellField | None = None, reps: int = 3, stream=None):
    """fpg_step_autotune: times one step of `params` under every launch shape
    (from a snapshot, restored afterwards; the counter does not advance) and
    keeps the fastest in the context; returns (best, all candidates)."""
    from .records import BatchTuning

    if wet_cells is not None:
        params.wet_cells = wet_cells.h.value
    n = lib.fpg_step_tuning_candidates(None, 0)
    res = (BatchTuning * n)()
    best = BatchTuning()
    check(lib.fpg_step_autotune(ctx.h, particles.h, met.h if met else None, pbl.h if pbl else None,
                                ctypes.byref(params), reps, res, n, ctypes.byref(best), stream), "fpg_step_autotune")
    return best.as_dict(), [r.as_dict() for r in res]


def get_step_tuning(ctx: Context) -> dict:
    from .records import BatchTuning

    t = BatchTuning()
    check(lib.fpg_step_get_tuning(ctx.h, ctypes.byref(t)), "fpg_step_get_tuning")
    return t.as_dict()


def set_step_tuning(ctx: Context, t: dict):
    from .records import BatchTuning

    bt = BatchTuning(t["block_threads"], t["min_blocks_per_sm"], t["particles_per_thread"], t.get("step_ms", 0.0))
    check(lib.fpg_step_set_tuning(ctx.h, ctypes.byref(bt)), "fpg_step_set_tuning")


def advect_dual_wind(ctx, particles, met, alpha, dt, xs=1.0, ys=1.0, zs=1.0):
    check(lib.fpg_advect_dual_wind(ctx.h, particles.h, met.h, alpha, dt, xs, ys, zs, None), "fpg_advect_dual_wind")


def langevin_fused(ctx, particles, pbl, dt, rho, n_substeps, min_height, key, counter):
    nxt = (ctypes.c_uint32 * 4)()
    check(lib.fpg_langevin_fused(ctx.h, particles.h, pbl.h, dt, rho, n_substeps, min_height, _u32arr(key, 2),
                                 _u32arr(counter, 4), nxt, None), "fpg_langevin_fused")
    return list(nxt)


def dry_deposition(ctx, particles, vdep: DeviceArray, dt, href, prob: DeviceArray | None = None):
    check(lib.fpg_dry_deposition(ctx.h, particles.h, _vp(vdep.ptr), dt, href, _vp(prob.ptr) if prob else None, None),
          "fpg_dry_deposition")


def wet_deposition(ctx, particles, lam: DeviceArray, frac: DeviceArray, dt, prob: DeviceArray | None = None):
    check(lib.fpg_wet_deposition(ctx.h, particles.h, _vp(lam.ptr), _vp(frac.ptr), dt,
                                 _vp(prob.ptr) if prob else None, None), "fpg_wet_deposition")


class Grid:
    def __init__(self, ctx: Context, nx: int, ny: int, nz: int):
        self.ctx, self.shape = ctx, (nx, ny, nz)
        h = _vp()
        check(lib.fpg_grid_create(ctx.h, nx, ny, nz, ctypes.byref(h)), "fpg_grid_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_grid_destroy(self.h)
        except Exception:
            pass

    def accumulate(self, particles: Particles, species: int = 0, mass_scale: float = 1.0e6, outheights=None,
                   stream=None):
        oh = None if outheights is None else np.ascontiguousarray(outheights, np.float32)
        check(lib.fpg_grid_accumulate(self.ctx.h, particles.h, self.h, species, mass_scale,
                                      None if oh is None else _p(oh), 0 if oh is None else oh.size, stream),
              "fpg_grid_accumulate")

    def cell_indices(self, particles: Particles, outheights=None) -> np.ndarray:
        n = particles.dispatch_count
        out = DeviceArray(self.ctx, n, np.uint32)
        oh = None if outheights is None else np.ascontiguousarray(outheights, np.float32)
        check(lib.fpg_grid_cell_indices(self.ctx.h, particles.h, self.h, None if oh is None else _p(oh),
                                        0 if oh is None else oh.size, _vp(out.ptr), None), "fpg_grid_cell_indices")
        return out.numpy()[:n]

    def download_async(self, counts_ptr: int | None, mass_ptr: int | None, stream=None):
        """Enqueue the copy of counts and scaled masses into host memory at the
        given addresses (page-locked for overlap) on `stream`, ordered after
        the last accumulate; returns at once (fpg_grid_download_async)."""
        check(lib.fpg_grid_download_async(self.h, _vp(counts_ptr) if counts_ptr else None,
                                          _vp(mass_ptr) if mass_ptr else None, stream), "fpg_grid_download_async")

    def download(self):
        n = self.shape[0] * self.shape[1] * self.shape[2]
        counts = np.empty(n, np.uint32)
        mass = np.empty(n, np.uint32)
        kg = np.empty(n, np.float32)
        check(lib.fpg_grid_download(self.h, _p(counts), _p(mass), _p(kg), None), "fpg_grid_download")
        return counts, mass, kg


class Compaction:
    def __init__(self, ctx: Context, capacity: int):
        self.ctx = ctx
        h = _vp()
        check(lib.fpg_compaction_create(ctx.h, capacity, ctypes.byref(h)), "fpg_compaction_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_compaction_destroy(self.h)
        except Exception:
            pass

    def compact(self, particles: Particles, indices: DeviceArray | None = None) -> int:
        cnt = ctypes.c_uint32()
        check(lib.fpg_compact(self.ctx.h, particles.h, self.h, ctypes.byref(cnt),
                              _vp(indices.ptr) if indices else None, None), "fpg_compact")
        return int(cnt.value)


class Sorter:
    """fpg_sorter: stable reorder of particles by 3-D met cell."""

    def __init__(self, ctx: Context, capacity: int):
        self.ctx = ctx
        h = _vp()
        check(lib.fpg_sorter_create(ctx.h, capacity, ctypes.byref(h)), "fpg_sorter_create")
        self.h = h

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                lib.fpg_sorter_destroy(self.h)
        except Exception:
            pass

    def sort(self, particles: Particles, met: Met, perm: DeviceArray | None = None, stream=None):
        check(lib.fpg_sort_by_cell(self.ctx.h, particles.h, met.h, self.h, _vp(perm.ptr) if perm else None, stream),
              "fpg_sort_by_cell")


def philox_uniforms(ctx: Context, key, counter, n_blocks: int):
    out = DeviceArray(ctx, 4 * n_blocks, np.float32)
    raw = DeviceArray(ctx, 4 * n_blocks, np.uint32)
    check(lib.fpg_philox_uniforms(ctx.h, _u32arr(key, 2), _u32arr(counter, 4), n_blocks, _vp(out.ptr),
                                  _vp(raw.ptr), None), "fpg_philox_uniforms")
    return out.numpy(), raw.numpy()


__all__ = [
    "Context", "DeviceArray", "Particles", "Met", "Pbl", "Surface", "CellField", "Grid", "Compaction",
    "pbl_diagnostics", "step", "advect_dual_wind", "langevin_fused", "dry_deposition", "wet_deposition",
    "philox_uniforms", "StepParams", "PblOptions", "_lib",
]
