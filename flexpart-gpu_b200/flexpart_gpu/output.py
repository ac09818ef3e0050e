"""Output formats fed from the device grids.

* ``write_gridded_output_netcdf``: the concentration/deposition snapshot of
  the reference's NetCDF writer (src/io/netcdf_output.rs:141-232): one file
  per snapshot, dimensions time(1), x, y, z, coordinate variables, the
  particle count and mass per concentration cell, dry and wet deposition per
  horizontal cell, and the same global and variable attributes.  The
  reference writes NetCDF-4 through libnetcdf; this image has no libnetcdf,
  so the file is NetCDF-3 (64-bit offset, scipy.io), which has no unsigned
  or 64-bit integer types: the u32 particle counts are stored as int32
  (checked to fit) and the i64 time as double (exact below 2^53 s).
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
                                dry_deposition_kg_m2=None, wet_deposition_kg_m2=None, dep_shape=None):
    """One snapshot: `counts` (u32) and `mass_kg` (f32) of nx*ny*nz cells in
    the grid's flat order ((ix*ny)+iy)*nz+iz; deposition grids of nx*ny cells
    in (ix*ny)+iy order (zeros when not given)."""
    from scipy.io import netcdf_file

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
    if counts.size and int(counts.max()) >= 2**31:
        raise OutputError("particle count per cell does not fit the file's int32")
    with netcdf_file(path, "w", version=2) as f:
        f.title = "FLEXPART-GPU concentration/deposition MVP output"
        f.source = "flexpart-gpu B200 backend"
        f.conventions = "CF-1.10"
        f.deterministic_fields = "true"
        f.species_index = np.int32(species_index)
        f.createDimension("time", 1)
        f.createDimension("x", nx)
        f.createDimension("y", ny)
        f.createDimension("z", nz)
        t = f.createVariable("time", "d", ("time",))
        t.units = "seconds since 1970-01-01 00:00:00 UTC"
        t[:] = np.array([time_seconds], np.float64)
        for name, n, axis in (("x", nx, "X"), ("y", ny, "Y"), ("z", nz, "Z")):
            v = f.createVariable(name, "f", (name,))
            v.axis = axis
            v[:] = np.arange(n, dtype=np.float32)
        c = f.createVariable("concentration_particle_count", "i", ("time", "x", "y", "z"))
        c.long_name = "particle count per concentration cell"
        c.units = "1"
        c[:] = counts.astype(np.int32).reshape(1, nx, ny, nz)
        m = f.createVariable("concentration_mass_kg", "f", ("time", "x", "y", "z"))
        m.long_name = "accumulated species mass per concentration cell"
        m.units = "kg"
        m[:] = mass_kg.reshape(1, nx, ny, nz)
        d = f.createVariable("dry_deposition_kg_m2", "f", ("time", "x", "y"))
        d.long_name = "dry deposition per horizontal cell"
        d.units = "kg m-2"
        d[:] = dry.reshape(1, nx, ny)
        w = f.createVariable("wet_deposition_kg_m2", "f", ("time", "x", "y"))
        w.long_name = "wet deposition per horizontal cell"
        w.units = "kg m-2"
        w[:] = wet.reshape(1, nx, ny)


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


__all__ = ["OutputError", "write_gridded_output_netcdf", "write_grid_netcdf", "validation_output",
           "write_validation_json"]
