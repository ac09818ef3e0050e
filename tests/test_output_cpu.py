"""Output formats (flexpart_gpu.output) on CPU: the NetCDF snapshot's
structure and values read back, the reference writer's validation errors
(src/io/netcdf_output.rs:60-120), and the validation artefact's host
recount agreeing with the oracle's gridding of the same particles."""
import numpy as np
import pytest

from flexpart_gpu import output, synthetic
from flexpart_gpu.records import GridDomain


def _grid():
    from oracle import orc

    scn = synthetic.config0()
    rec = synthetic.particles_at_sources(scn, 5_000, seed=4)
    st = orc.State.from_records(rec)
    counts, mass, _ = orc.grid(st, len(rec), 0, 1e6, scn.outheights, scn.out_shape)
    return scn, rec, counts, mass.astype(np.float32) / np.float32(1e6)


def test_netcdf_snapshot_round_trip(tmp_path):
    from scipy.io import netcdf_file

    scn, _, counts, kg = _grid()
    nx, ny, nz = scn.out_shape
    dry = np.linspace(0, 1, nx * ny, dtype=np.float32)
    path = tmp_path / "snap.nc"
    output.write_gridded_output_netcdf(path, counts, kg, scn.out_shape, 1_704_070_800, 0, dry_deposition_kg_m2=dry)
    with netcdf_file(path, "r", mmap=False) as f:
        assert f.dimensions == {"time": 1, "x": nx, "y": ny, "z": nz}
        assert f.conventions == b"CF-1.10" and f.species_index == 0
        assert f.variables["time"][0] == 1_704_070_800
        assert f.variables["time"].units == b"seconds since 1970-01-01 00:00:00 UTC"
        assert np.array_equal(f.variables["x"][:], np.arange(nx, dtype=np.float32))
        c = f.variables["concentration_particle_count"][:]
        assert c.shape == (1, nx, ny, nz) and np.array_equal(c.reshape(-1), counts.astype(np.int32))
        assert np.array_equal(f.variables["concentration_mass_kg"][:].reshape(-1), kg)
        assert f.variables["concentration_mass_kg"].units == b"kg"
        assert np.array_equal(f.variables["dry_deposition_kg_m2"][:].reshape(-1), dry)
        assert not f.variables["wet_deposition_kg_m2"][:].any()
        assert f.variables["wet_deposition_kg_m2"].units == b"kg m-2"


def test_netcdf_writer_validation_errors(tmp_path):
    scn, _, counts, kg = _grid()
    nx, ny, nz = scn.out_shape
    with pytest.raises(output.OutputError, match="non-zero"):
        output.write_gridded_output_netcdf(tmp_path / "a.nc", [], [], (0, ny, nz), 0)
    with pytest.raises(output.OutputError, match="horizontal shape mismatch"):
        output.write_gridded_output_netcdf(tmp_path / "b.nc", counts, kg, scn.out_shape, 0, dep_shape=(nx, ny + 1))
    with pytest.raises(output.OutputError, match="length mismatch"):
        output.write_gridded_output_netcdf(tmp_path / "c.nc", counts[:-1], kg, scn.out_shape, 0)


def test_validation_artefact_host_recount_matches_the_oracle_grid(tmp_path):
    import json

    scn, rec, counts, kg = _grid()
    m = scn.met
    dom = GridDomain(m.xlon0, m.ylat0, m.dx_deg, m.dy_deg, m.nx, m.ny)
    out = output.validation_output(rec, counts, kg, dom, scn.out_shape, scn.outheights, total_steps=3)
    assert out["particle_count_per_cell_host_gridding"] == out["particle_count_per_cell"]
    assert out["total_particles_active"] == len(rec) and out["total_steps"] == 3
    assert out["grid"]["nx"] == scn.out_shape[0] and out["grid"]["heights_m"] == list(scn.outheights)
    assert out["particle_z_stats"]["count"] == len(rec)
    path = tmp_path / "v.json"
    output.write_validation_json(path, particles=rec, counts_device=counts, mass_kg=kg, domain=dom,
                                 shape=scn.out_shape, outheights=scn.outheights, total_steps=3)
    assert json.load(open(path))["total_steps"] == 3
