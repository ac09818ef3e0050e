"""CPU checks of the boundary: the library loads without a GPU and exports
every function include/fpg.h declares; calls without a device fail with a
status, not a crash."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for hdr in ("fpg.h", "fpg_driver.h"):
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
    assert set(_lib.EXPORTED) | set(_lib.EXPORTED_DRIVER) == declared


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
