"""ctypes view of the parity oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline leg of bench.py, always as the checker.  The product
package never imports this module.

`State` holds a particle population as structure-of-arrays in float32 (the
parity build) or float64 (the FP64 error reference).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
_PKG = os.path.join(_ROOT, "flexpart-gpu_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from flexpart_gpu.records import (  # noqa: E402
    PARTICLE_DTYPE,
    SURFACE_DTYPE,
    PblOptions,
    StepParams,
)

LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


def _ptr(a, t=ctypes.c_void_p):
    if a is None:
        return None
    return ctypes.cast(a.ctypes.data, t)


class _StateF32(ctypes.Structure):
    _fields_ = [
        ("cell_x", _i32p), ("cell_y", _i32p),
        ("pos_x", _f32p), ("pos_y", _f32p), ("pos_z", _f32p),
        ("flags", _u32p),
        ("mass", _f32p * 4),
        ("vel_u", _f32p), ("vel_v", _f32p), ("vel_w", _f32p),
        ("turb_u", _f32p), ("turb_v", _f32p), ("turb_w", _f32p),
        ("cbt", _i32p),
    ]


class _StateF64(ctypes.Structure):
    _fields_ = [
        ("cell_x", _i32p), ("cell_y", _i32p),
        ("pos_x", _f64p), ("pos_y", _f64p), ("pos_z", _f64p),
        ("flags", _u32p),
        ("mass", _f64p * 4),
        ("vel_u", _f64p), ("vel_v", _f64p), ("vel_w", _f64p),
        ("turb_u", _f64p), ("turb_v", _f64p), ("turb_w", _f64p),
        ("cbt", _i32p),
    ]


class _PblF32(ctypes.Structure):
    _fields_ = [("ustar", _f32p), ("wstar", _f32p), ("hmix", _f32p), ("oli", _f32p),
                ("nx", ctypes.c_size_t), ("ny", ctypes.c_size_t)]


class _PblF64(ctypes.Structure):
    _fields_ = [("ustar", _f64p), ("wstar", _f64p), ("hmix", _f64p), ("oli", _f64p),
                ("nx", ctypes.c_size_t), ("ny", ctypes.c_size_t)]


_REAL_FIELDS = ["pos_x", "pos_y", "pos_z", "vel_u", "vel_v", "vel_w", "turb_u", "turb_v", "turb_w"]


class State:
    """Particle SoA for the oracle.  `mass` is (4, n)."""

    def __init__(self, n: int, dtype=np.float32):
        self.n = n
        self.dtype = np.dtype(dtype)
        self.cell_x = np.zeros(n, np.int32)
        self.cell_y = np.zeros(n, np.int32)
        self.flags = np.zeros(n, np.uint32)
        self.cbt = np.zeros(n, np.int32)
        for f in _REAL_FIELDS:
            setattr(self, f, np.zeros(n, self.dtype))
        self.mass = np.zeros((4, n), self.dtype)

    @classmethod
    def from_records(cls, rec: np.ndarray, dtype=np.float32) -> "State":
        s = cls(len(rec), dtype)
        for f in ("cell_x", "cell_y", "flags", "cbt"):
            getattr(s, f)[:] = rec[f]
        for f in _REAL_FIELDS:
            getattr(s, f)[:] = rec[f]
        s.mass[:] = rec["mass"].T
        return s

    def to_records(self) -> np.ndarray:
        rec = np.zeros(self.n, PARTICLE_DTYPE)
        for f in ("cell_x", "cell_y", "flags", "cbt"):
            rec[f] = getattr(self, f)
        for f in _REAL_FIELDS:
            rec[f] = getattr(self, f).astype(np.float32)
        rec["mass"] = self.mass.T.astype(np.float32)
        return rec

    def copy(self) -> "State":
        s = State(self.n, self.dtype)
        for f in ("cell_x", "cell_y", "flags", "cbt", "mass") + tuple(_REAL_FIELDS):
            getattr(s, f)[:] = getattr(self, f)
        return s

    def astype(self, dtype) -> "State":
        s = State(self.n, dtype)
        for f in ("cell_x", "cell_y", "flags", "cbt", "mass") + tuple(_REAL_FIELDS):
            getattr(s, f)[:] = getattr(self, f)
        return s

    def grid_x(self):
        return self.cell_x.astype(np.float64) + self.pos_x.astype(np.float64)

    def grid_y(self):
        return self.cell_y.astype(np.float64) + self.pos_y.astype(np.float64)

    def cstruct(self):
        f64 = self.dtype == np.float64
        S = _StateF64 if f64 else _StateF32
        rp = _f64p if f64 else _f32p
        st = S()
        st.cell_x = _ptr(self.cell_x, _i32p)
        st.cell_y = _ptr(self.cell_y, _i32p)
        st.flags = _ptr(self.flags, _u32p)
        st.cbt = _ptr(self.cbt, _i32p)
        for f in _REAL_FIELDS:
            setattr(st, f, _ptr(getattr(self, f), rp))
        for k in range(4):
            st.mass[k] = ctypes.cast(self.mass[k].ctypes.data, rp)
        return st


def _sfx(dtype):
    return "_f64" if np.dtype(dtype) == np.float64 else "_f32"


# ---- scalar functions ------------------------------------------------------

def philox(counter, key):
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in counter])
    k = (ctypes.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (ctypes.c_uint32 * 4)()
    lib.orc_philox4x32_10(c, k, o)
    return list(o)


def counter_add(counter, offset):
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in counter])
    o = (ctypes.c_uint32 * 4)()
    lib.orc_counter_add_u64(c, ctypes.c_uint64(offset), o)
    return list(o)


def next_counter(counter, particle_count, n_substeps):
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in counter])
    o = (ctypes.c_uint32 * 4)()
    lib.orc_next_counter(c, ctypes.c_uint64(particle_count), ctypes.c_uint32(n_substeps), o)
    return list(o)


def philox_uniforms(key, counter, n_blocks):
    out = np.zeros(4 * n_blocks, np.float32)
    raw = np.zeros(4 * n_blocks, np.uint32)
    k = (ctypes.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in counter])
    lib.orc_philox_uniforms(k, c, ctypes.c_size_t(n_blocks), _ptr(out), _ptr(raw))
    return out, raw


def u32_to_uniform01(v):
    lib.orc_u32_to_uniform01.restype = ctypes.c_float
    return lib.orc_u32_to_uniform01(ctypes.c_uint32(v))


def _ctype(dtype):
    return ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float


def box_muller(u0, u1, dtype=np.float32):
    t = _ctype(dtype)
    out = (t * 2)()
    getattr(lib, "orc_box_muller" + _sfx(dtype))(t(u0), t(u1), out)
    return out[0], out[1]


HANNA_FIELDS = ["ust", "wst", "ol", "h", "zeta", "sigu", "sigv", "sigw", "dsigwdz", "dsigw2dz",
                "tlu", "tlv", "tlw"]


def hanna(ust, wst, ol, h, z, dtype=np.float32):
    t = _ctype(dtype)
    out = (t * 13)()
    getattr(lib, "orc_hanna" + _sfx(dtype))(t(ust), t(wst), t(ol), t(h), t(z), out)
    return dict(zip(HANNA_FIELDS, list(out)))


def hanna_short_w(ust, wst, ol, h, z, dtype=np.float32):
    t = _ctype(dtype)
    out = (t * 3)()
    getattr(lib, "orc_hanna_short_w" + _sfx(dtype))(t(ust), t(wst), t(ol), t(h), t(z), out)
    return tuple(out)


def obukhov_from_inverse(oli, dtype=np.float32):
    t = _ctype(dtype)
    f = getattr(lib, "orc_obukhov_from_inverse" + _sfx(dtype))
    f.restype = t
    return f(t(oli))


def langevin_h(prev, sigma, tl, dt, eta, dtype=np.float32):
    t = _ctype(dtype)
    f = getattr(lib, "orc_langevin_h" + _sfx(dtype))
    f.restype = t
    return f(t(prev), t(sigma), t(tl), t(dt), t(eta))


def langevin_v(prev, sigw, tlw, dsigwdz, dt, rho, eta, dtype=np.float32):
    t = _ctype(dtype)
    f = getattr(lib, "orc_langevin_v" + _sfx(dtype))
    f.restype = t
    return f(t(prev), t(sigw), t(tlw), t(dsigwdz), t(dt), t(rho), t(eta))


def trilinear(field, x, y, z, dtype=np.float32):
    field = np.ascontiguousarray(field, np.float32)
    nx, ny, nz = field.shape
    t = _ctype(dtype)
    f = getattr(lib, "orc_trilinear" + _sfx(dtype))
    f.restype = t
    return f(_ptr(field), ctypes.c_size_t(nx), ctypes.c_size_t(ny), ctypes.c_size_t(nz),
             t(x), t(y), t(z))


def meters_to_level(heights, z, dtype=np.float32):
    h = np.ascontiguousarray(heights, np.float32)
    t = _ctype(dtype)
    f = getattr(lib, "orc_meters_to_level" + _sfx(dtype))
    f.restype = t
    return f(_ptr(h), ctypes.c_size_t(len(h)), t(z))


def advect_cpu(state: State, u, v, w, dt, scale=(1.0, 1.0, 1.0)):
    """advect_particle_cpu over all slots (physics/advection.rs:100-153)."""
    u = np.ascontiguousarray(u, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    nx, ny, nz = u.shape
    t = _ctype(state.dtype)
    getattr(lib, "orc_advect_cpu" + _sfx(state.dtype))(
        ctypes.c_size_t(state.n), _ptr(state.cell_x), _ptr(state.cell_y), _ptr(state.pos_x),
        _ptr(state.pos_y), _ptr(state.pos_z), _ptr(state.flags), _ptr(state.vel_u),
        _ptr(state.vel_v), _ptr(state.vel_w), _ptr(u), _ptr(v), _ptr(w),
        ctypes.c_size_t(nx), ctypes.c_size_t(ny), ctypes.c_size_t(nz),
        t(dt), t(scale[0]), t(scale[1]), t(scale[2]))


def dry_survival(vdep, dt, href, dtype=np.float32):
    t = _ctype(dtype)
    f = getattr(lib, "orc_dry_survival" + _sfx(dtype))
    f.restype = t
    return f(t(vdep), t(dt), t(href))


def wet_probability(lam, dt, frac, dtype=np.float32):
    t = _ctype(dtype)
    f = getattr(lib, "orc_wet_probability" + _sfx(dtype))
    f.restype = t
    return f(t(lam), t(dt), t(frac))


def wet_cell(lsp, convp, cc, a, b):
    lam = ctypes.c_float()
    fr = ctypes.c_float()
    lib.orc_wet_cell(ctypes.c_float(lsp), ctypes.c_float(convp), ctypes.c_float(cc),
                     ctypes.c_float(a), ctypes.c_float(b), ctypes.byref(lam), ctypes.byref(fr))
    return lam.value, fr.value


def wet_cells(lsp, convp, cc, a, b):
    lsp = np.ascontiguousarray(lsp, np.float32).ravel()
    convp = None if convp is None else np.ascontiguousarray(convp, np.float32).ravel()
    cc = None if cc is None else np.ascontiguousarray(cc, np.float32).ravel()
    lam = np.zeros_like(lsp)
    fr = np.zeros_like(lsp)
    lib.orc_wet_cells_grid(ctypes.c_size_t(lsp.size), _ptr(lsp), _ptr(convp), _ptr(cc), ctypes.c_float(a),
                           ctypes.c_float(b), _ptr(lam), _ptr(fr))
    return lam, fr


def lerp_field(a, b, t, threads=0):
    """Whole-field time lerp of the reference's CPU pipeline
    (interpolate_wind_field_linear, io/temporal.rs:67-120)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    out = np.empty_like(a)
    lib.orc_lerp_field(ctypes.c_size_t(a.size), _ptr(a), _ptr(b), ctypes.c_float(t), _ptr(out),
                       ctypes.c_int(threads or (os.cpu_count() or 1)))
    return out


# ---- grid functions --------------------------------------------------------

class Pbl:
    def __init__(self, nx, ny, dtype=np.float32):
        self.nx, self.ny, self.dtype = nx, ny, np.dtype(dtype)
        for f in ("ustar", "wstar", "hmix", "oli", "sshf", "ssr", "surfstr"):
            setattr(self, f, np.zeros(nx * ny, self.dtype))

    def cstruct(self):
        f64 = self.dtype == np.float64
        S = _PblF64 if f64 else _PblF32
        rp = _f64p if f64 else _f32p
        s = S()
        for f in ("ustar", "wstar", "hmix", "oli"):
            setattr(s, f, _ptr(getattr(self, f), rp))
        s.nx, s.ny = self.nx, self.ny
        return s


def pbl_diagnostics(surface_t0, surface_t1, alpha, nx, ny, options=None, dtype=np.float32):
    """Per-cell surface lerp + PBL diagnostics (pbl_diagnostics.wgsl)."""
    options = options or PblOptions.default()
    s0 = np.ascontiguousarray(surface_t0, SURFACE_DTYPE)
    s1 = np.ascontiguousarray(surface_t1, SURFACE_DTYPE)
    pbl = Pbl(nx, ny, dtype)
    t = _ctype(dtype)
    getattr(lib, "orc_pbl_grid" + _sfx(dtype))(
        _ptr(s0), _ptr(s1), ctypes.c_size_t(nx * ny), t(alpha), ctypes.byref(options),
        _ptr(pbl.ustar), _ptr(pbl.wstar), _ptr(pbl.hmix), _ptr(pbl.oli), _ptr(pbl.sshf),
        _ptr(pbl.ssr), _ptr(pbl.surfstr))
    return pbl


def step(state: State, n, met, pbl: Pbl, params: StepParams, wet_cells_lf=None, wet_shape=None,
         threads=0, dry_velocity=None, wet_lambda=None, wet_fraction=None,
         dry_prob=None, wet_prob=None, wind_bias=None, rng_index=None):
    """The fused production step over slots [0, n).  `met` is a dict with
    u0, v0, w0, u1, v1, w1 ((nx, ny, nz) float32) and heights (nz,).
    `rng_index` (uint32, n) gives each slot's Philox block index when the
    state is a sample of a larger population (default: the slot itself)."""
    u0 = np.ascontiguousarray(met["u0"], np.float32)
    nx, ny, nz = u0.shape
    arrs = [u0] + [np.ascontiguousarray(met[k], np.float32) for k in ("v0", "w0", "u1", "v1", "w1")]
    hts = np.ascontiguousarray(met["heights"], np.float32)
    prm = StepParams()
    ctypes.pointer(prm)[0] = params
    keep = []
    for name, arr in (("dry_velocity_dev", dry_velocity), ("wet_lambda_dev", wet_lambda),
                      ("wet_fraction_dev", wet_fraction), ("dry_probability_dev", dry_prob),
                      ("wet_probability_dev", wet_prob)):
        if arr is not None:
            assert arr.dtype == np.float32 and arr.flags.c_contiguous
            keep.append(arr)
            setattr(prm, name, arr.ctypes.data)
        else:
            setattr(prm, name, None)
    prm.wet_cells = None
    lam = fr = None
    wnx = wny = 1
    if wet_cells_lf is not None:
        lam = np.ascontiguousarray(wet_cells_lf[0], np.float32)
        fr = np.ascontiguousarray(wet_cells_lf[1], np.float32)
        wnx, wny = wet_shape
    threads = threads or (os.cpu_count() or 1)
    st = state.cstruct()
    pc = pbl.cstruct() if pbl is not None else (_PblF64 if state.dtype == np.float64 else _PblF32)()
    bias = None if wind_bias is None else np.ascontiguousarray(wind_bias, np.float64).reshape(-1)
    assert bias is None or bias.size == 3 * nx * ny * nz
    idx = None if rng_index is None else np.ascontiguousarray(rng_index, np.uint32)
    assert idx is None or idx.size >= n
    getattr(lib, "orc_step_indexed" + _sfx(state.dtype))(
        ctypes.byref(st), ctypes.c_size_t(n), *[_ptr(a) for a in arrs],
        ctypes.c_size_t(nx), ctypes.c_size_t(ny), ctypes.c_size_t(nz), _ptr(hts),
        ctypes.byref(pc), ctypes.byref(prm), _ptr(lam), _ptr(fr),
        ctypes.c_size_t(wnx), ctypes.c_size_t(wny), ctypes.c_int(threads), _ptr(bias), _ptr(idx))


def level_of(z, outheights, dtype=np.float32):
    h = np.ascontiguousarray(outheights, np.float32)
    t = _ctype(dtype)
    f = getattr(lib, "orc_level_of" + _sfx(dtype))
    f.restype = ctypes.c_uint32
    return f(t(z), _ptr(h), ctypes.c_size_t(len(h)))


def grid(state: State, n, species, mass_scale, outheights, shape):
    nx, ny, nz = shape
    counts = np.zeros(nx * ny * nz, np.uint32)
    mass = np.zeros(nx * ny * nz, np.uint32)
    cells = np.zeros(max(n, 1), np.uint32)
    oh = np.zeros(nz, np.float32) if outheights is None else np.ascontiguousarray(outheights, np.float32)
    t = _ctype(state.dtype)
    st = state.cstruct()
    getattr(lib, "orc_grid" + _sfx(state.dtype))(
        ctypes.byref(st), ctypes.c_size_t(n), ctypes.c_uint32(species), t(mass_scale), _ptr(oh),
        ctypes.c_size_t(nx), ctypes.c_size_t(ny), ctypes.c_size_t(nz), _ptr(counts), _ptr(mass),
        _ptr(cells))
    return counts, mass, cells[:n]


def compaction_indices(flags):
    flags = np.ascontiguousarray(flags, np.uint32)
    idx = np.zeros(max(len(flags), 1), np.uint32)
    lib.orc_compaction_indices.restype = ctypes.c_uint32
    count = lib.orc_compaction_indices(_ptr(flags), ctypes.c_size_t(len(flags)), _ptr(idx))
    return int(count), idx[:count]


def compact_records(rec: np.ndarray):
    """compaction.wgsl passes 1-4 on fpg_particle records: returns
    (compacted records, active count, indices)."""
    count, idx = compaction_indices(rec["flags"])
    out = rec.copy()
    out[:count] = rec[idx]
    out["flags"][count:] = rec["flags"][count:] & ~np.uint32(1)
    return out, count, idx


def cell_keys(state: State, n, heights, shape):
    """Met-cell keys of the spatial reorder (inactive: nx*ny*nz)."""
    nx, ny, nz = shape
    h = np.ascontiguousarray(heights, np.float32)
    keys = np.zeros(max(n, 1), np.uint32)
    getattr(lib, "orc_cell_keys" + _sfx(state.dtype))(
        ctypes.c_size_t(n), _ptr(state.cell_x), _ptr(state.cell_y), _ptr(state.pos_x), _ptr(state.pos_y),
        _ptr(state.pos_z), _ptr(state.flags), _ptr(h), ctypes.c_size_t(nx), ctypes.c_size_t(ny),
        ctypes.c_size_t(nz), _ptr(keys))
    return keys[:n]


def sort_by_cell(rec: np.ndarray, n, heights, shape):
    """Stable reorder of records [0, n) by met-cell key; returns (records, perm)."""
    keys = cell_keys(State.from_records(rec[:n]), n, heights, shape)
    perm = np.argsort(keys, kind="stable").astype(np.uint32)
    out = rec.copy()
    out[:n] = rec[:n][perm]
    return out, perm


def interpolation_alpha(t0, t1, target, clamp=True):
    out = ctypes.c_float()
    st = lib.orc_interpolation_alpha(ctypes.c_int64(t0), ctypes.c_int64(t1), ctypes.c_int64(target),
                                     ctypes.c_int32(1 if clamp else 0), ctypes.byref(out))
    return st, out.value


def parse_timestamp(s: str):
    out = ctypes.c_int64()
    st = lib.orc_parse_timestamp(s.encode(), ctypes.byref(out))
    return st, out.value


def target_emitted_count(particle_count, start, end, now, released):
    lib.orc_target_emitted_count.restype = ctypes.c_uint64
    return lib.orc_target_emitted_count(ctypes.c_uint64(particle_count), ctypes.c_int64(start),
                                        ctypes.c_int64(end), ctypes.c_int64(now),
                                        ctypes.c_uint64(released))


def sample_stratified(bounds, idx, total):
    b = (ctypes.c_double * 6)(*bounds)
    o = (ctypes.c_double * 3)()
    lib.orc_sample_stratified(b, ctypes.c_uint64(idx), ctypes.c_uint64(total), o)
    return tuple(o)


def geo_to_relative(lon, lat, domain):
    d = (ctypes.c_double * 6)(*domain)
    cx, cy = ctypes.c_int32(), ctypes.c_int32()
    fx, fy = ctypes.c_float(), ctypes.c_float()
    st = lib.orc_geo_to_relative(ctypes.c_double(lon), ctypes.c_double(lat), d, ctypes.byref(cx),
                                 ctypes.byref(cy), ctypes.byref(fx), ctypes.byref(fy))
    return st, cx.value, cy.value, fx.value, fy.value


# ---- CBL skewed PDF and convective mixing (physics/cbl.rs, physics/convection.rs)

CBL_PDF_FIELDS = ["updraft_weight", "updraft_mean_m_s", "updraft_sigma_m_s", "downdraft_weight",
                  "downdraft_mean_m_s", "downdraft_sigma_m_s", "second_moment_w2", "third_moment_w3", "skewness",
                  "transition", "z_over_h"]

lib.orc_cbl_transition_factor.restype = ctypes.c_float
lib.orc_cbl_transition_factor.argtypes = [ctypes.c_float, ctypes.c_float]
lib.orc_cbl_probability_density.restype = ctypes.c_float
lib.orc_cbl_probability_density.argtypes = [_f32p, ctypes.c_float]
lib.orc_cbl_sample.restype = ctypes.c_float
lib.orc_cbl_sample.argtypes = [_f32p, ctypes.c_float, ctypes.c_float, ctypes.c_float]
lib.orc_cbl_branch_constrained.restype = ctypes.c_float
lib.orc_cbl_branch_constrained.argtypes = [_f32p, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32]
lib.orc_cbl_infer_branch.restype = ctypes.c_int32
lib.orc_cbl_infer_branch.argtypes = [ctypes.c_float, ctypes.c_int32]
lib.orc_level_index_from_height.restype = ctypes.c_size_t
lib.orc_level_index_from_height.argtypes = [_f32p, ctypes.c_size_t, ctypes.c_float]
lib.orc_convection_chain.restype = ctypes.c_int32
lib.orc_convection_chain.argtypes = [_f32p, ctypes.c_size_t, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_int32, ctypes.c_float, ctypes.c_float, _f32p, _f32p, _f32p]


def cbl_transition_factor(h, ol):
    return lib.orc_cbl_transition_factor(h, ol)


def cbl_pdf(z, h, wstar, sigma_w, ol) -> np.ndarray:
    """compute_cbl_bigaussian_pdf: the 11 floats of CBL_PDF_FIELDS."""
    inp = np.array([z, h, wstar, sigma_w, ol], np.float32)
    out = np.zeros(11, np.float32)
    lib.orc_cbl_pdf(_ptr(inp), _ptr(out))
    return out


def cbl_reconstruct_moments(pdf) -> np.ndarray:
    pdf = np.ascontiguousarray(pdf, np.float32)
    out = np.zeros(3, np.float32)
    lib.orc_cbl_reconstruct_moments(_ptr(pdf), _ptr(out))
    return out


def cbl_probability_density(pdf, w) -> float:
    pdf = np.ascontiguousarray(pdf, np.float32)
    return lib.orc_cbl_probability_density(_ptr(pdf, _f32p), w)


def cbl_sample(pdf, branch_uniform, u0, u1) -> float:
    pdf = np.ascontiguousarray(pdf, np.float32)
    return lib.orc_cbl_sample(_ptr(pdf, _f32p), branch_uniform, u0, u1)


def cbl_sample_stream(pdf, key, counter, n) -> np.ndarray:
    """n successive sample_cbl_vertical_velocity_with_rng draws."""
    pdf = np.ascontiguousarray(pdf, np.float32)
    k = np.array(key, np.uint32)
    c = np.array(counter, np.uint32)
    out = np.zeros(n, np.float32)
    lib.orc_cbl_sample_stream(_ptr(pdf), _ptr(k), _ptr(c), ctypes.c_size_t(n), _ptr(out))
    return out


def cbl_infer_branch(previous_w, time_direction) -> str:
    return "updraft" if lib.orc_cbl_infer_branch(previous_w, time_direction) else "downdraft"


def cbl_branch_constrained(pdf, branch, u0, u1, time_direction) -> float:
    pdf = np.ascontiguousarray(pdf, np.float32)
    return lib.orc_cbl_branch_constrained(_ptr(pdf, _f32p), 1 if branch == "updraft" else 0, u0, u1, time_direction)


def cbl_sample_slots(rec, hanna16, inputs) -> np.ndarray:
    """The CBL dispatch over records: (n, 12) = sample + PDF, zeros inactive."""
    n = rec.size
    flags = np.ascontiguousarray(rec["flags"], np.uint32)
    z = np.ascontiguousarray(rec["pos_z"], np.float32)
    h = np.ascontiguousarray(hanna16.view(np.float32).reshape(n, 16) if hanna16.dtype.names else hanna16,
                             np.float32)
    i4 = np.ascontiguousarray(inputs.view(np.float32).reshape(n, 4) if inputs.dtype.names else inputs, np.float32)
    out = np.zeros((max(n, 1), 12), np.float32)
    lib.orc_cbl_sample_slots(ctypes.c_size_t(n), _ptr(flags), _ptr(z), _ptr(h), _ptr(i4), _ptr(out))
    return out[:n]


def hanna_params_slots(rec, ustar, wstar, hmix, oli, pnx, pny) -> np.ndarray:
    """compute_hanna_params_gpu over records: (n, 16) HannaParams floats."""
    n = rec.size
    cols = {k: np.ascontiguousarray(rec[k]) for k in ("cell_x", "cell_y", "pos_x", "pos_y", "pos_z", "flags")}
    f = [np.ascontiguousarray(a, np.float32).reshape(-1) for a in (ustar, wstar, hmix, oli)]
    out = np.zeros((max(n, 1), 16), np.float32)
    lib.orc_hanna_params_slots(ctypes.c_size_t(n), _ptr(cols["cell_x"]), _ptr(cols["cell_y"]), _ptr(cols["pos_x"]),
                               _ptr(cols["pos_y"]), _ptr(cols["pos_z"]), _ptr(cols["flags"]), _ptr(f[0]),
                               _ptr(f[1]), _ptr(f[2]), _ptr(f[3]), ctypes.c_size_t(pnx), ctypes.c_size_t(pny),
                               _ptr(out))
    return out[:n]


def level_index_from_height(iface, height) -> int:
    iface = np.ascontiguousarray(iface, np.float32)
    return int(lib.orc_level_index_from_height(_ptr(iface, _f32p), iface.size, height))


def convection_chain(iface, precip, wstar, hbl, cape_override, dt):
    """(status, matrix (L, L) column-major as [source, destination],
    detrainment weights, info dict)."""
    iface = np.ascontiguousarray(iface, np.float32)
    L = max(iface.size - 1, 1)
    m = np.zeros(L * L, np.float32)
    det = np.zeros(L, np.float32)
    info = np.zeros(6, np.float32)
    st = lib.orc_convection_chain(_ptr(iface, _f32p), iface.size, precip, wstar, hbl,
                                  0 if cape_override is None else 1,
                                  0.0 if cape_override is None else cape_override, dt, _ptr(m, _f32p),
                                  _ptr(det, _f32p), _ptr(info, _f32p))
    keys = ["is_active", "cape_j_kg", "cloud_base_level", "cloud_top_level", "convective_timescale_s",
            "mixing_fraction"]
    return st, m, det, dict(zip(keys, info.tolist()))


def convective_mixing(rec, matrix, iface):
    """apply_convective_mixing_to_particles_cpu on a copy of the records."""
    out = rec.copy()
    iface = np.ascontiguousarray(iface, np.float32)
    L = iface.size - 1
    centers = (np.float32(0.5) * (iface[:-1] + iface[1:])).astype(np.float32)
    flags = np.ascontiguousarray(out["flags"])
    z = np.ascontiguousarray(out["pos_z"])
    cbt = np.ascontiguousarray(out["cbt"])
    m = np.ascontiguousarray(matrix, np.float32)
    lib.orc_convective_mixing(ctypes.c_size_t(out.size), _ptr(flags), _ptr(z), _ptr(cbt), _ptr(m),
                              ctypes.c_size_t(L), _ptr(iface), _ptr(centers))
    out["pos_z"] = z
    out["cbt"] = cbt
    return out
