"""CPU checks of the boundary: the library loads without a GPU and exports
every function include/fpg.h declares; calls without a device fail with a
status, not a crash."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for hdr in ("fpg.h", "fpg_driver.h", "fpg_adjoint.h"):
        txt = open(os.path.join(ROOT, "include", hdr)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(fpg_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    from flexpart_gpu import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) | set(_lib.EXPORTED_DRIVER) | set(_lib.EXPORTED_ADJOINT) == declared


def test_status_strings_and_version():
    from flexpart_gpu import _lib
    assert _lib.lib.fpg_abi_version() == 1
    assert _lib.lib.fpg_status_string(-2) == b"invalid time step"
    assert _lib.lib.fpg_status_string(0) == b"ok"


def test_null_handles_are_rejected():
    from flexpart_gpu import _lib
    lib = _lib.lib
    assert lib.fpg_step(None, None, None, None, None, None, None) == -1
    assert lib.fpg_particles_upload(None, 0, 0, None, None) == -1
    assert lib.fpg_grid_download(None, None, None, None, None) == -1
    # the driver's timing and validation switches
    assert lib.fpg_forward_set_profiling(None, 1) == -1
    assert lib.fpg_forward_last_timing(None, None) == -1
    assert lib.fpg_forward_set_validation_mode(None, 1) == -1
    assert lib.fpg_backward_set_validation_mode(None, 1) == -1


def test_record_layouts_match_the_c_header(tmp_path):
    """Every ctypes record the host side passes through the ABI has the size
    and field offsets the C compiler gives the header's struct."""
    import ctypes
    import shutil
    import subprocess

    from flexpart_gpu import records as R

    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    pairs = {
        "fpg_step_params": R.StepParams, "fpg_pbl_options": R.PblOptions, "fpg_release": R.Release,
        "fpg_grid_domain": R.GridDomain, "fpg_forward_config": R.ForwardConfig, "fpg_met_bracket": R.MetBracket,
        "fpg_forcing": R.Forcing, "fpg_step_report": R.StepReport, "fpg_batch_scenario": R.BatchScenario,
        "fpg_batch_tuning": R.BatchTuning, "fpg_receptor": R.Receptor,
        "fpg_receptor_release": R.ReceptorRelease, "fpg_source_region": R.SourceRegion,
        "fpg_source_collection": R.SourceCollection, "fpg_backward_config": R.BackwardConfig,
        "fpg_inverse_config": R.InverseConfig,
        "fpg_batch_config": R.BatchConfig, "fpg_convection_inputs": R.ConvectionInputs,
        "fpg_convection_column": R.ConvectionColumn, "fpg_step_timing": R.StepTiming,
    }
    dtypes = {"fpg_hanna_params": R.HANNA_PARAMS_DTYPE, "fpg_cbl_sampling_input": R.CBL_INPUT_DTYPE,
              "fpg_cbl_sampling_output": R.CBL_OUTPUT_DTYPE, "fpg_particle": R.PARTICLE_DTYPE,
              "fpg_surface_cell": R.SURFACE_DTYPE}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fpg_adjoint.h"', "int main(void) {"]
    for c, py in pairs.items():
        lines.append(f'printf("{c} size %zu\\n", sizeof({c}));')
        for name, _ in py._fields_:
            lines.append(f'printf("{c} {name} %zu\\n", offsetof({c}, {name}));')
    for c, dt in dtypes.items():
        lines.append(f'printf("{c} size %zu\\n", sizeof({c}));')
        for name in dt.names:
            lines.append(f'printf("{c} {name} %zu\\n", offsetof({c}, {name}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(ROOT, "include")
    subprocess.run([gcc, "-I", str(inc), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        c, name, v = line.split()
        got[(c, name)] = int(v)
    for c, py in pairs.items():
        assert got[(c, "size")] == ctypes.sizeof(py), c
        for name, _ in py._fields_:
            assert got[(c, name)] == getattr(py, name).offset, (c, name)
    for c, dt in dtypes.items():
        assert got[(c, "size")] == dt.itemsize, c
        for name in dt.names:
            assert got[(c, name)] == dt.fields[name][1], (c, name)


def test_batch_tuning_candidates_listed_without_a_device():
    from flexpart_gpu.batch import tuning_candidates

    c = tuning_candidates()
    assert len(c) >= 4
    shapes = {(t["block_threads"], t["min_blocks_per_sm"], t["particles_per_thread"]) for t in c}
    assert (256, 4, 1) in shapes
    assert len(shapes) == len(c)


def test_step_tuning_candidates_listed_without_a_device():
    from flexpart_gpu import api
    from flexpart_gpu import _lib

    c = api.step_tuning_candidates()
    shapes = [(t["block_threads"], t["min_blocks_per_sm"], t["particles_per_thread"]) for t in c]
    assert shapes[0] == (256, 5, 1) and len(set(shapes)) == len(shapes) >= 4
    lib = _lib.lib
    assert lib.fpg_step_autotune(None, None, None, None, None, 1, None, 0, None, None) == -1
    assert lib.fpg_step_set_tuning(None, None) == -1
    assert lib.fpg_step_get_tuning(None, None) == -1


def test_missing_library_fails_loudly(tmp_path):
    """No CPU fallback: without libfpg.so the package does not import."""
    import subprocess
    import sys

    code = ("import sys; sys.path.insert(0, %r)\n"
            "try:\n"
            "    import flexpart_gpu.api\n"
            "except ImportError as e:\n"
            "    print('refused:', e)\n"
            "    sys.exit(0)\n"
            "sys.exit(3)\n") % os.path.join(ROOT, "flexpart-gpu_b200")
    env = dict(os.environ, FPG_LIBRARY=str(tmp_path / "absent" / "libfpg.so"))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "no CPU fallback" in r.stdout
