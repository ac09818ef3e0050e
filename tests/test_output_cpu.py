"""Output formats (flexpart_gpu.output) on CPU: the NetCDF snapshot's
structure, types and values read back (CDF-5 by the module's reader, the
64-bit offset variant by scipy), the CDF-5 header against its grammar, the
reference writer's validation errors (src/io/netcdf_output.rs:60-120), and
the validation artefact's host recount agreeing with the oracle's gridding
of the same particles."""
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
    """The default CDF-5 file read back: the reference's dimensions,
    attributes and variable types (i64 time, u32 counts, f32 masses)."""
    scn, _, counts, kg = _grid()
    nx, ny, nz = scn.out_shape
    dry = np.linspace(0, 1, nx * ny, dtype=np.float32)
    path = tmp_path / "snap.nc"
    output.write_gridded_output_netcdf(path, counts, kg, scn.out_shape, 1_704_070_800, 0, dry_deposition_kg_m2=dry)
    assert open(path, "rb").read(4) == b"CDF\x05"
    f = output.read_netcdf(path)
    assert f["format"] == "cdf5"
    assert f["dimensions"] == {"time": 1, "x": nx, "y": ny, "z": nz}
    assert f["attributes"]["conventions"] == "CF-1.10" and f["attributes"]["species_index"].tolist() == [0]
    v = f["variables"]
    assert v["time"]["data"].dtype == np.int64 and v["time"]["data"].tolist() == [1_704_070_800]
    assert v["time"]["attributes"]["units"] == "seconds since 1970-01-01 00:00:00 UTC"
    assert np.array_equal(v["x"]["data"], np.arange(nx, dtype=np.float32)) and v["x"]["attributes"]["axis"] == "X"
    c = v["concentration_particle_count"]
    assert c["dimensions"] == ("time", "x", "y", "z") and c["data"].dtype == np.uint32
    assert c["data"].shape == (1, nx, ny, nz) and np.array_equal(c["data"].reshape(-1), counts.astype(np.uint32))
    assert v["concentration_mass_kg"]["data"].dtype == np.float32
    assert np.array_equal(v["concentration_mass_kg"]["data"].reshape(-1), kg)
    assert v["concentration_mass_kg"]["attributes"]["units"] == "kg"
    assert np.array_equal(v["dry_deposition_kg_m2"]["data"].reshape(-1), dry)
    assert not v["wet_deposition_kg_m2"]["data"].any()
    assert v["wet_deposition_kg_m2"]["attributes"]["units"] == "kg m-2"


def test_netcdf_counts_above_int32_need_cdf5(tmp_path):
    counts = np.array([0, 2**31 + 5, 2**32 - 1, 7], np.uint32)
    kg = np.ones(4, np.float32)
    output.write_gridded_output_netcdf(tmp_path / "a.nc", counts, kg, (2, 2, 1), 0)
    got = output.read_netcdf(tmp_path / "a.nc")["variables"]["concentration_particle_count"]["data"]
    assert np.array_equal(got.reshape(-1), counts)
    with pytest.raises(output.OutputError, match="int32"):
        output.write_gridded_output_netcdf(tmp_path / "b.nc", counts, kg, (2, 2, 1), 0, fmt="cdf2")


def test_netcdf_cdf2_snapshot_reads_in_scipy(tmp_path):
    """The 64-bit offset variant through an independent reader (scipy.io)."""
    from scipy.io import netcdf_file

    scn, _, counts, kg = _grid()
    nx, ny, nz = scn.out_shape
    dry = np.linspace(0, 1, nx * ny, dtype=np.float32)
    path = tmp_path / "snap2.nc"
    output.write_gridded_output_netcdf(path, counts, kg, scn.out_shape, 1_704_070_800, 0, dry_deposition_kg_m2=dry,
                                       fmt="cdf2")
    with netcdf_file(path, "r", mmap=False) as f:
        assert f.version_byte == 2
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
    # and the reader on the same file
    g = output.read_netcdf(path)
    assert g["format"] == "cdf2"
    assert np.array_equal(g["variables"]["concentration_particle_count"]["data"].reshape(-1), counts.astype(np.int32))


def test_netcdf_reader_on_files_scipy_wrote(tmp_path):
    from scipy.io import netcdf_file

    for version in (1, 2):
        path = tmp_path / f"s{version}.nc"
        with netcdf_file(path, "w", version=version) as f:
            f.title = "abc"
            f.n = np.int32(5)
            f.createDimension("a", 3)
            f.createDimension("b", 2)
            v = f.createVariable("v", "h", ("a", "b"))
            v[:] = np.arange(6, dtype=np.int16).reshape(3, 2)
            v.units = "m"
            w = f.createVariable("w", "d", ("b",))
            w[:] = [1.5, -2.5]
            w.scale = np.float32(0.25)
            b = f.createVariable("k", "b", ("a",))
            b[:] = np.array([-1, 0, 1], np.int8)
        r = output.read_netcdf(path)
        assert r["format"] == f"cdf{version}"
        assert r["dimensions"] == {"a": 3, "b": 2}
        assert r["attributes"]["title"] == "abc" and r["attributes"]["n"].tolist() == [5]
        assert r["variables"]["v"]["data"].tolist() == [[0, 1], [2, 3], [4, 5]]
        assert r["variables"]["v"]["attributes"] == {"units": "m"}
        assert r["variables"]["w"]["data"].tolist() == [1.5, -2.5]
        assert r["variables"]["w"]["attributes"]["scale"].tolist() == [0.25]
        assert r["variables"]["k"]["data"].tolist() == [-1, 0, 1]


def test_netcdf_cdf5_header_bytes():
    """A one-variable CDF-5 file against its bytes assembled from the
    format's grammar: magic, 64-bit numrecs, the dimension list, one text
    global attribute, one u32 variable with a 64-bit dimension id, size and
    begin, then the data padded to 4 bytes."""
    import os
    import tempfile

    def i32(n):
        return n.to_bytes(4, "big")

    def i64(n):
        return n.to_bytes(8, "big")

    head = (b"CDF\x05" + i64(0)
            + i32(10) + i64(1) + i64(1) + b"d\0\0\0" + i64(3)            # dimension d = 3
            + i32(12) + i64(1) + i64(2) + b"ab\0\0" + i32(2) + i64(3) + b"xyz\0"   # ab = "xyz"
            + i32(11) + i64(1) + i64(1) + b"v\0\0\0" + i64(1) + i64(0)    # variable v(d)
            + i32(0) + i64(0) + i32(9) + i64(12))                             # no attributes, NC_UINT, 12 B
    begin = len(head) + 8
    want = head + i64(begin) + i32(1) + i32(2**32 - 1) + i32(7)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "t.nc")
        output.write_netcdf(path, [("d", 3)], [("v", ("d",), np.array([1, 2**32 - 1, 7], np.uint32), [])],
                            [("ab", "xyz")])
        assert open(path, "rb").read() == want
        assert output.read_netcdf(path)["variables"]["v"]["data"].tolist() == [1, 2**32 - 1, 7]


def test_netcdf_types_the_classic_formats_lack_are_refused(tmp_path):
    with pytest.raises(output.OutputError, match="cdf2"):
        output.write_netcdf(tmp_path / "a.nc", [("d", 2)], [("v", ("d",), np.zeros(2, np.uint32), [])], fmt="cdf2")
    with pytest.raises(output.OutputError, match="unknown"):
        output.write_netcdf(tmp_path / "b.nc", [("d", 2)], [], fmt="hdf5")


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
