"""Output formats fed from the device grids.

* ``write_gridded_output_netcdf``: the concentration/deposition snapshot of
  the reference's NetCDF writer (src/io/netcdf_output.rs:141-232): one file
  per snapshot, dimensions time(1), x, y, z, coordinate variables, the
  particle count and mass per concentration cell, dry and wet deposition per
  horizontal cell, the same global and variable attributes and the same
  variable types (i64 time, f32 coordinates, u32 counts, f32 masses).  The
  reference writes NetCDF-4 (HDF5) through libnetcdf, which this image does
  not have; the file here is the netCDF 64-bit data format (CDF-5), which
  holds those types and which libnetcdf (4.4 and later) reads through the
  same API, written by this module.  ``fmt="cdf2"`` gives the 64-bit offset
  format for readers without CDF-5 (scipy.io): counts as int32 (checked to
  fit) and time as double (exact below 2^53 s).
* ``read_netcdf``: the reader of those files (CDF-1, CDF-2, CDF-5).
* ``validation_output``: the JSON artefact of the reference's validation
  run (src/bin/fortran-validation.rs:60-94): grid description, device and
  host-recounted particle counts per cell, mass per cell, active count,
  step count and particle height / position statistics.
"""
from __future__ import annotations

import json

import numpy as np


class OutputError(ValueError):
    """NetcdfOutputError (src/io/netcdf_output.rs:60-82)."""


# ---- NetCDF classic-family files (CDF-1, CDF-2, CDF-5) ----------------------
# The header grammar of the netCDF classic formats and of the 64-bit data
# format (CDF-5, netCDF-C >= 4.4 and PnetCDF read it): magic "CDF" + version
# byte, the record count, then the dimension, global attribute and variable
# lists, each a 32-bit tag and a count; names, attribute values and
# variable data padded to 4 bytes; everything big-endian.  CDF-5 widens every
# count, length, dimension id and size to 64 bits and adds the unsigned and
# 64-bit integer types, which the reference's variables use (u32 particle
# counts, i64 time).
_TAG_DIM, _TAG_VAR, _TAG_ATT = 10, 11, 12
_NC_CHAR = 2
_NC_TYPE_OF = {np.dtype(np.int8): 1, np.dtype(np.int16): 3, np.dtype(np.int32): 4, np.dtype(np.float32): 5,
               np.dtype(np.float64): 6, np.dtype(np.uint8): 7, np.dtype(np.uint16): 8, np.dtype(np.uint32): 9,
               np.dtype(np.int64): 10, np.dtype(np.uint64): 11}
_DTYPE_OF = {1: ">i1", 2: "S1", 3: ">i2", 4: ">i4", 5: ">f4", 6: ">f8", 7: ">u1", 8: ">u2", 9: ">u4",
             10: ">i8", 11: ">u8"}
_CDF1_TYPES = {1, 2, 3, 4, 5, 6}
_VERSIONS = {"cdf1": 1, "cdf2": 2, "cdf5": 5}


def _pad4(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 4)


class _Header:
    def __init__(self, version):
        self.v = version
        self.parts = []

    def count(self, n):      # NON_NEG: 32-bit in CDF-1/2, 64-bit in CDF-5
        self.parts.append(int(n).to_bytes(8 if self.v == 5 else 4, "big"))

    def i32(self, n):
        self.parts.append(int(n).to_bytes(4, "big"))

    def offset(self, n):     # OFFSET: 32-bit in CDF-1, 64-bit in CDF-2/5
        self.parts.append(int(n).to_bytes(4 if self.v == 1 else 8, "big"))

    def name(self, s):
        b = s.encode("utf-8")
        self.count(len(b))
        self.parts.append(_pad4(b))

    def attrs(self, atts):
        if not atts:
            self.i32(0)
            self.count(0)
            return
        self.i32(_TAG_ATT)
        self.count(len(atts))
        for k, val in atts:
            self.name(k)
            if isinstance(val, str):
                b = val.encode("utf-8")
                self.i32(_NC_CHAR)
                self.count(len(b))
                self.parts.append(_pad4(b))
            else:
                a = np.atleast_1d(np.asarray(val))
                t = _NC_TYPE_OF[a.dtype]
                if self.v != 5 and t not in _CDF1_TYPES:
                    raise OutputError(f"attribute `{k}`: type {a.dtype} needs the CDF-5 format")
                self.i32(t)
                self.count(a.size)
                self.parts.append(_pad4(a.astype(_DTYPE_OF[t]).tobytes()))

    def bytes(self):
        return b"".join(self.parts)


def write_netcdf(path, dims, variables, global_attrs=(), fmt: str = "cdf5"):
    """A netCDF file of fixed-size dimensions (`dims`: (name, length) pairs)
    and variables (`variables`: (name, dimension names, array, attribute
    pairs)) in the classic (`cdf1`), 64-bit offset (`cdf2`) or 64-bit data
    (`cdf5`) format; each array is stored in its own dtype."""
    if fmt not in _VERSIONS:
        raise OutputError(f"unknown netCDF format `{fmt}` (cdf1, cdf2, cdf5)")
    v = _VERSIONS[fmt]
    dim_ids = {n: i for i, (n, _) in enumerate(dims)}
    lens = dict(dims)
    prepared = []
    for name, dnames, data, atts in variables:
        a = np.asarray(data)
        t = _NC_TYPE_OF.get(a.dtype)
        if t is None or (v != 5 and t not in _CDF1_TYPES):
            raise OutputError(f"variable `{name}`: type {a.dtype} is not storable in the {fmt} format")
        shape = tuple(lens[d] for d in dnames)
        if a.size != int(np.prod(shape, dtype=np.int64)):
            raise OutputError(f"variable `{name}`: {a.size} values for shape {shape}")
        raw = _pad4(np.ascontiguousarray(a.reshape(shape)).astype(_DTYPE_OF[t]).tobytes())
        prepared.append((name, dnames, t, atts, raw))

    def header(begins):
        h = _Header(v)
        h.parts.append(b"CDF" + bytes([v]))
        h.count(0)                                   # numrecs: no record dimension
        h.i32(_TAG_DIM)
        h.count(len(dims))
        for n, length in dims:
            if length <= 0:
                raise OutputError(f"dimension `{n}` must be non-zero, got {length}")
            h.name(n)
            h.count(length)
        h.attrs(list(global_attrs))
        h.i32(_TAG_VAR if prepared else 0)
        h.count(len(prepared))
        for (name, dnames, t, atts, raw), b in zip(prepared, begins):
            h.name(name)
            h.count(len(dnames))
            for d in dnames:
                h.count(dim_ids[d])
            h.attrs(list(atts))
            h.i32(t)
            vsize = len(raw)
            if v != 5 and vsize >= 2**32 - 4:
                vsize = 2**32 - 1                    # the classic formats' marker for a large variable
            h.count(vsize)
            h.offset(b)
        return h.bytes()

    size = len(header([0] * len(prepared)))
    begins, at = [], size
    for p in prepared:
        begins.append(at)
        at += len(p[4])
    if v == 1 and at >= 2**31:
        raise OutputError("file too large for the classic format; use cdf2 or cdf5")
    with open(path, "wb") as f:
        f.write(header(begins))
        for p in prepared:
            f.write(p[4])


class _Reader:
    def __init__(self, buf):
        self.b = buf
        self.at = 0

    def take(self, n):
        s = self.b[self.at:self.at + n]
        if len(s) != n:
            raise OutputError("truncated netCDF header")
        self.at += n
        return s

    def i32(self):
        return int.from_bytes(self.take(4), "big")

    def count(self):
        return int.from_bytes(self.take(8 if self.v == 5 else 4), "big")

    def offset(self):
        return int.from_bytes(self.take(4 if self.v == 1 else 8), "big")

    def name(self):
        n = self.count()
        s = self.take(n + (-n % 4))[:n]
        return s.decode("utf-8")

    def attrs(self):
        tag, n = self.i32(), self.count()
        if tag not in (0, _TAG_ATT) or (tag == 0 and n):
            raise OutputError("malformed attribute list")
        out = {}
        for _ in range(n):
            k = self.name()
            t, m = self.i32(), self.count()
            dt = np.dtype(_DTYPE_OF[t])
            raw = self.take(m * dt.itemsize + (-(m * dt.itemsize) % 4))[:m * dt.itemsize]
            out[k] = raw.decode("utf-8") if t == _NC_CHAR else np.frombuffer(raw, dt).astype(dt.newbyteorder("="))
        return out


def read_netcdf(path):
    """The dimensions, global attributes and variables of a classic-family
    netCDF file (CDF-1, CDF-2 or CDF-5) without a record dimension:
    {"format", "dimensions": {name: length}, "attributes": {...},
    "variables": {name: {"dimensions", "data" (native byte order),
    "attributes"}}}.  Text attributes come back as str, numeric ones as
    arrays."""
    buf = open(path, "rb").read()
    r = _Reader(buf)
    magic = r.take(4)
    if magic[:3] != b"CDF" or magic[3] not in (1, 2, 5):
        raise OutputError(f"not a classic-family netCDF file: {magic!r}")
    r.v = magic[3]
    if r.count() != 0:
        raise OutputError("record variables are not read")
    tag, n = r.i32(), r.count()
    dims = []
    for _ in range(n):
        dims.append((r.name(), r.count()))
    gatts = r.attrs()
    tag, n = r.i32(), r.count()
    variables = {}
    for _ in range(n):
        name = r.name()
        ids = [r.count() for _ in range(r.count())]
        atts = r.attrs()
        t = r.i32()
        r.count()                                    # vsize
        begin = r.offset()
        dt = np.dtype(_DTYPE_OF[t])
        shape = tuple(dims[i][1] for i in ids)
        m = int(np.prod(shape, dtype=np.int64))
        data = np.frombuffer(buf, dt, count=m, offset=begin).reshape(shape).astype(dt.newbyteorder("="))
        variables[name] = {"dimensions": tuple(dims[i][0] for i in ids), "data": data, "attributes": atts}
    return {"format": {1: "cdf1", 2: "cdf2", 5: "cdf5"}[r.v], "dimensions": dict(dims), "attributes": gatts,
            "variables": variables}


def _validate(counts, mass_kg, shape, dry, wet, dep_shape):
    nx, ny, nz = shape
    if nx == 0 or ny == 0 or nz == 0:
        raise OutputError(f"concentration shape must be non-zero, got {shape}")
    dnx, dny = dep_shape
    if dnx == 0 or dny == 0:
        raise OutputError(f"deposition shape must be non-zero, got {dep_shape}")
    if (nx, ny) != (dnx, dny):
        raise OutputError(f"concentration/deposition horizontal shape mismatch: concentration=({nx},{ny}), "
                          f"deposition=({dnx},{dny})")
    for name, a, n in (("concentration.particle_count_per_cell", counts, nx * ny * nz),
                       ("concentration.concentration_mass_kg", mass_kg, nx * ny * nz),
                       ("deposition.dry_deposition_kg_m2", dry, nx * ny),
                       ("deposition.wet_deposition_kg_m2", wet, nx * ny)):
        if np.asarray(a).size != n:
            raise OutputError(f"length mismatch for `{name}`: expected {n}, got {np.asarray(a).size}")


def write_gridded_output_netcdf(path, counts, mass_kg, shape, time_seconds: int, species_index: int = 0,
                                dry_deposition_kg_m2=None, wet_deposition_kg_m2=None, dep_shape=None,
                                fmt: str = "cdf5"):
    """One snapshot: `counts` (u32) and `mass_kg` (f32) of nx*ny*nz cells in
    the grid's flat order ((ix*ny)+iy)*nz+iz; deposition grids of nx*ny cells
    in (ix*ny)+iy order (zeros when not given)."""
    nx, ny, nz = shape
    dep_shape = (nx, ny) if dep_shape is None else tuple(dep_shape)
    dry = np.zeros(dep_shape[0] * dep_shape[1], np.float32) if dry_deposition_kg_m2 is None \
        else np.asarray(dry_deposition_kg_m2, np.float32).reshape(-1)
    wet = np.zeros(dep_shape[0] * dep_shape[1], np.float32) if wet_deposition_kg_m2 is None \
        else np.asarray(wet_deposition_kg_m2, np.float32).reshape(-1)
    counts = np.asarray(counts).reshape(-1)
    mass_kg = np.asarray(mass_kg, np.float32).reshape(-1)
    _validate(counts, mass_kg, shape, dry, wet, dep_shape)
    if not (0 <= species_index < 2**31):
        raise OutputError(f"species index does not fit i32: {species_index}")
    if fmt == "cdf5":
        counts_out = counts.astype(np.uint32)
        time_out = np.array([time_seconds], np.int64)
    else:
        if counts.size and int(counts.max()) >= 2**31:
            raise OutputError(f"particle count per cell does not fit the {fmt} file's int32")
        counts_out = counts.astype(np.int32)
        time_out = np.array([time_seconds], np.float64)
    dims = [("time", 1), ("x", nx), ("y", ny), ("z", nz)]
    gatts = [("title", "FLEXPART-GPU concentration/deposition MVP output"),
             ("source", "flexpart-gpu B200 backend"),
             ("conventions", "CF-1.10"),
             ("deterministic_fields", "true"),
             ("species_index", np.int32(species_index))]
    variables = [
        ("time", ("time",), time_out, [("units", "seconds since 1970-01-01 00:00:00 UTC")]),
        ("x", ("x",), np.arange(nx, dtype=np.float32), [("axis", "X")]),
        ("y", ("y",), np.arange(ny, dtype=np.float32), [("axis", "Y")]),
        ("z", ("z",), np.arange(nz, dtype=np.float32), [("axis", "Z")]),
        ("concentration_particle_count", ("time", "x", "y", "z"), counts_out,
         [("long_name", "particle count per concentration cell"), ("units", "1")]),
        ("concentration_mass_kg", ("time", "x", "y", "z"), mass_kg,
         [("long_name", "accumulated species mass per concentration cell"), ("units", "kg")]),
        ("dry_deposition_kg_m2", ("time", "x", "y"), dry,
         [("long_name", "dry deposition per horizontal cell"), ("units", "kg m-2")]),
        ("wet_deposition_kg_m2", ("time", "x", "y"), wet,
         [("long_name", "wet deposition per horizontal cell"), ("units", "kg m-2")]),
    ]
    write_netcdf(path, dims, variables, gatts, fmt)


def write_grid_netcdf(path, grid, time_seconds: int, species_index: int = 0, **kw):
    """A device Grid (flexpart_gpu.api.Grid) written as one snapshot."""
    counts, _, kg = grid.download()
    write_gridded_output_netcdf(path, counts, kg, grid.shape, time_seconds, species_index, **kw)


def validation_output(particles: np.ndarray, counts_device, mass_kg, domain, shape, outheights, total_steps: int):
    """The reference's validation artefact (fortran-validation.rs:60-94) as a
    dict: the device's counts and masses per cell beside counts recomputed on
    the host from the particle records (nearest cell, first level whose
    height is >= z, the top level above), plus the particles' height and
    position statistics."""
    nx, ny, nz = shape
    act = (particles["flags"] & 1) != 0
    p = particles[act]
    oh = np.asarray(outheights, np.float32)
    ix = np.clip(p["cell_x"], 0, nx - 1).astype(np.int64)
    iy = np.clip(p["cell_y"], 0, ny - 1).astype(np.int64)
    if oh.size and oh[-1] > 0:
        iz = np.minimum(np.searchsorted(oh, p["pos_z"], side="left"), nz - 1)
    else:
        iz = np.clip(np.floor(p["pos_z"]).astype(np.int64), 0, nz - 1)
    host = np.bincount((ix * ny + iy) * nz + iz, minlength=nx * ny * nz).astype(np.uint32)
    out = {
        "grid": {"nx": nx, "ny": ny, "nz": nz, "dx": float(domain.dx), "dy": float(domain.dy),
                 "xlon0": float(domain.xlon0), "ylat0": float(domain.ylat0),
                 "heights_m": [float(h) for h in oh]},
        "particle_count_per_cell": [int(c) for c in np.asarray(counts_device).reshape(-1)],
        "particle_count_per_cell_host_gridding": [int(c) for c in host],
        "concentration_mass_kg": [float(m) for m in np.asarray(mass_kg, np.float32).reshape(-1)],
        "total_particles_active": int(act.sum()),
        "total_steps": int(total_steps),
        "particle_z_stats": None,
    }
    if p.size:
        z = p["pos_z"].astype(np.float32)
        lon = domain.xlon0 + (p["cell_x"].astype(np.float64) + p["pos_x"].astype(np.float64)) * domain.dx
        lat = domain.ylat0 + (p["cell_y"].astype(np.float64) + p["pos_y"].astype(np.float64)) * domain.dy
        out["particle_z_stats"] = {
            "count": int(z.size), "min_m": float(z.min()), "max_m": float(z.max()), "mean_m": float(z.mean()),
            "std_m": float(z.std()), "lon_mean": float(lon.mean()), "lat_mean": float(lat.mean()),
            "lon_std": float(lon.std()), "lat_std": float(lat.std()),
        }
    return out


def write_validation_json(path, **kw):
    with open(path, "w") as f:
        json.dump(validation_output(**kw), f)


__all__ = ["OutputError", "write_gridded_output_netcdf", "write_grid_netcdf", "write_netcdf", "read_netcdf",
           "validation_output", "write_validation_json"]
