"""ctypes binding of libfpg.so (include/fpg.h).

The library is the only compute path: importing this module raises if the
built library is missing, and nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes
import os

from .records import PblOptions, StepParams

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("FPG_LIBRARY", os.path.join(_PKG_ROOT, "lib", "libfpg.so"))


class FpgError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = lib.fpg_status_string(status).decode() if lib is not None else str(status)
        extra = ""
        if status == -100:
            extra = f" (cudaError {lib.fpg_last_cuda_error()})"
        super().__init__(f"{what}: {msg} [{status}]{extra}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libfpg.so not found at {LIB_PATH}; build it with `make -C flexpart-gpu_b200` "
            "(there is no CPU fallback)")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_i32 = ctypes.c_int32
_u32 = ctypes.c_uint32
_f32 = ctypes.c_float
_u32p = ctypes.POINTER(ctypes.c_uint32)


def _sig(name, restype, *argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_sig("fpg_status_string", ctypes.c_char_p, _i32)
_sig("fpg_last_cuda_error", _i32)
_sig("fpg_abi_version", _i32)
_sig("fpg_ctx_create", _i32, _i32, ctypes.POINTER(_vp))
_sig("fpg_ctx_destroy", _i32, _vp)
_sig("fpg_ctx_stream", _vp, _vp)
_sig("fpg_ctx_synchronize", _i32, _vp, _vp)
_sig("fpg_ctx_kernel_launches", ctypes.c_uint64, _vp)
_sig("fpg_device_alloc", _i32, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_device_free", _i32, _vp, _vp)
_sig("fpg_memcpy", _i32, _vp, _vp, _vp, _sz, _i32, _vp)
_sig("fpg_memset", _i32, _vp, _vp, _i32, _sz, _vp)
_sig("fpg_particles_create", _i32, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_particles_destroy", _i32, _vp)
_sig("fpg_particles_capacity", _sz, _vp)
_sig("fpg_particles_dispatch_count", _sz, _vp)
_sig("fpg_particles_set_dispatch_count", _i32, _vp, _sz)
_sig("fpg_particles_upload", _i32, _vp, _sz, _sz, _vp, _vp)
_sig("fpg_particles_upload_slots", _i32, _vp, _vp, _sz, _vp, _vp)
_sig("fpg_particles_download", _i32, _vp, _sz, _sz, _vp, _vp)
_sig("fpg_particles_field", _vp, _vp, _i32)
_sig("fpg_particles_copy_field", _i32, _vp, _i32, _sz, _sz, _vp, _i32, _vp)
_sig("fpg_met_create", _i32, _vp, _sz, _sz, _sz, ctypes.POINTER(_vp))
_sig("fpg_met_destroy", _i32, _vp)
_sig("fpg_met_upload_frame", _i32, _vp, _i32, _vp, _vp, _vp, _vp)
_sig("fpg_met_upload_frame_device", _i32, _vp, _i32, _vp, _vp, _vp, _vp)
_sig("fpg_met_upload_bracket_device", _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_met_set_level_heights", _i32, _vp, _vp, _sz)
_sig("fpg_pbl_create", _i32, _vp, _sz, _sz, ctypes.POINTER(_vp))
_sig("fpg_pbl_destroy", _i32, _vp)
_sig("fpg_pbl_upload", _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_pbl_download", _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_surface_create", _i32, _vp, _sz, _sz, ctypes.POINTER(_vp))
_sig("fpg_surface_destroy", _i32, _vp)
_sig("fpg_surface_upload", _i32, _vp, _i32, _vp, _vp)
_sig("fpg_pbl_diagnostics", _i32, _vp, _vp, _f32, ctypes.POINTER(PblOptions), _vp, _vp)
_sig("fpg_cellfield_create", _i32, _vp, _sz, _sz, ctypes.POINTER(_vp))
_sig("fpg_cellfield_destroy", _i32, _vp)
_sig("fpg_cellfield_upload", _i32, _vp, _vp, _vp, _vp)
_sig("fpg_cellfield_from_precipitation", _i32, _vp, _vp, _vp, _vp, _f32, _f32, _vp)
_sig("fpg_step_params_default", None, ctypes.POINTER(StepParams))
_sig("fpg_step", _i32, _vp, _vp, _vp, _vp, ctypes.POINTER(StepParams), _u32p, _vp)
_sig("fpg_step_tuning_candidates", _u32, _vp, _u32)
_sig("fpg_step_autotune", _i32, _vp, _vp, _vp, _vp, ctypes.POINTER(StepParams), _u32, _vp, _u32, _vp, _vp)
_sig("fpg_step_set_tuning", _i32, _vp, _vp)
_sig("fpg_step_get_tuning", _i32, _vp, _vp)
_sig("fpg_advect_dual_wind", _i32, _vp, _vp, _vp, _f32, _f32, _f32, _f32, _f32, _vp)
_sig("fpg_langevin_fused", _i32, _vp, _vp, _vp, _f32, _f32, _u32, _f32, _u32p, _u32p, _u32p, _vp)
_sig("fpg_dry_deposition", _i32, _vp, _vp, _vp, _f32, _f32, _vp, _vp)
_sig("fpg_wet_deposition", _i32, _vp, _vp, _vp, _vp, _f32, _vp, _vp)
_sig("fpg_grid_create", _i32, _vp, _sz, _sz, _sz, ctypes.POINTER(_vp))
_sig("fpg_grid_destroy", _i32, _vp)
_sig("fpg_grid_accumulate", _i32, _vp, _vp, _vp, _u32, _f32, _vp, _sz, _vp)
_sig("fpg_grid_cell_indices", _i32, _vp, _vp, _vp, _vp, _sz, _vp, _vp)
_sig("fpg_grid_download", _i32, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_grid_counts_device", _vp, _vp)
_sig("fpg_grid_mass_device", _vp, _vp)
_sig("fpg_compaction_create", _i32, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_compaction_destroy", _i32, _vp)
_sig("fpg_compact", _i32, _vp, _vp, _vp, _u32p, _vp, _vp)
_sig("fpg_philox_uniforms", _i32, _vp, _u32p, _u32p, _sz, _vp, _vp, _vp)
_sig("fpg_compaction_indices_static", _i32, _vp, _vp, _sz, _vp, _vp, _vp)
_sig("fpg_dispatch_hanna_params", _i32, _vp, _vp, _vp, _vp, _sz, _vp)
_sig("fpg_grid_download_async", _i32, _vp, _vp, _vp, _vp)
_sig("fpg_langevin_with_hanna", _i32, _vp, _vp, _vp, _sz, _f32, _f32, _u32, _f32, _u32p, _u32p, _u32p, _vp)
_sig("fpg_cbl_sample", _i32, _vp, _vp, _vp, _sz, _vp, _sz, _vp, _vp)
_sig("fpg_cbl_sample_philox", _i32, _vp, _vp, _vp, _u32p, _u32p, _vp, _vp)
_sig("fpg_convection_build_chain", _i32, _vp, _f32, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_convection_level_index", _sz, _vp, _sz, _f32)
_sig("fpg_convection_apply_profile", _i32, _vp, _sz, _vp, _sz, _vp)
_sig("fpg_convection_create", _i32, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_convection_destroy", _i32, _vp)
_sig("fpg_convection_set_matrix", _i32, _vp, _vp, _sz, _vp, _sz, _vp)
_sig("fpg_convection_heights", _i32, _vp, _vp)
_sig("fpg_convective_mixing", _i32, _vp, _vp, _vp, _vp)
_sig("fpg_forward_config_default", None, _vp)
_sig("fpg_parse_timestamp", _i32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64))
_sig("fpg_forward_create", _i32, _vp, _vp, _vp, _sz, _vp, _sz, _sz, _sz, _sz, _vp, ctypes.POINTER(_vp))
_sig("fpg_forward_destroy", _i32, _vp)
_sig("fpg_forward_has_remaining_steps", _i32, _vp)
_sig("fpg_forward_current_time", ctypes.c_int64, _vp)
_sig("fpg_forward_run_timestep", _i32, _vp, _vp, _vp, _vp)
_sig("fpg_forward_finalize", _i32, _vp)
_sig("fpg_forward_particles", _vp, _vp)
_sig("fpg_forward_accumulate_grid", _i32, _vp, _vp, _u32, _f32, _vp, _sz)
_sig("fpg_batch_create", _i32, _vp, _vp, _vp, _sz, _sz, _sz, _sz, _vp, ctypes.POINTER(_vp))
_sig("fpg_batch_destroy", _i32, _vp)
_sig("fpg_batch_upload_frame", _i32, _vp, _u32, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_batch_run", _i32, _vp, _u32, _i32)
_sig("fpg_batch_run_sequential", _i32, _vp, _u32)
_sig("fpg_batch_steps_done", ctypes.c_uint64, _vp)
_sig("fpg_batch_scenario_slots", _i32, _vp, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_sz))
_sig("fpg_batch_particles", _vp, _vp)
_sig("fpg_batch_download_grids", _i32, _vp, _vp, _vp)
_sig("fpg_batch_errors", _i32, _vp, ctypes.POINTER(_i32))
_sig("fpg_batch_tuning_candidates", _u32, _vp, _u32)
_sig("fpg_batch_autotune", _i32, _vp, _u32, _vp, _u32, _vp)
_sig("fpg_batch_set_tuning", _i32, _vp, _vp)
_sig("fpg_batch_get_tuning", _i32, _vp, _vp)
_sig("fpg_inverse_create", _i32, _vp, _vp, _vp, _vp, _sz, _sz, _sz, _sz, _vp, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_inverse_destroy", _i32, _vp)
_sig("fpg_inverse_upload_frame", _i32, _vp, _u32, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_inverse_set_sources", _i32, _vp, _vp, _vp)
_sig("fpg_inverse_set_wind_bias", _i32, _vp, _vp)
_sig("fpg_inverse_forward", _i32, _vp, _vp)
_sig("fpg_inverse_backward", _i32, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_inverse_batch", _vp, _vp)
_sig("fpg_inverse_device_bytes", ctypes.c_uint64, _vp)
_sig("fpg_backward_config_default", None, _vp)
_sig("fpg_backward_create", _i32, _vp, _vp, _vp, _sz, _vp, _sz, _vp, _sz, _sz, _sz, _sz, _vp, ctypes.POINTER(_vp))
_sig("fpg_backward_destroy", _i32, _vp)
_sig("fpg_backward_has_remaining_steps", _i32, _vp)
_sig("fpg_backward_current_time", ctypes.c_int64, _vp)
_sig("fpg_backward_run_timestep", _i32, _vp, _vp, _vp, _vp, _vp)
_sig("fpg_backward_particles", _vp, _vp)
_sig("fpg_backward_set_validation_mode", _i32, _vp, _i32)
_sig("fpg_forward_met_ring", _i32, _vp, _u32)
_sig("fpg_forward_prefetch_frame", _i32, _vp, ctypes.c_int64, _vp, _vp, _vp, _vp)
_sig("fpg_forward_met_ring_stats", _i32, _vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64))
_sig("fpg_forward_set_profiling", _i32, _vp, _i32)
_sig("fpg_forward_set_validation_mode", _i32, _vp, _i32)
_sig("fpg_forward_last_timing", _i32, _vp, _vp)
_sig("fpg_host_alloc", _i32, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_host_free", _i32, _vp, _vp)
_sig("fpg_sorter_create", _i32, _vp, _sz, ctypes.POINTER(_vp))
_sig("fpg_sorter_destroy", _i32, _vp)
_sig("fpg_sort_by_cell", _i32, _vp, _vp, _vp, _vp, _vp, _vp)


def check(status: int, what: str) -> None:
    if status != 0:
        raise FpgError(status, what)


# Every symbol include/fpg.h declares (checked by the CPU test suite).
EXPORTED = [
    "fpg_status_string", "fpg_last_cuda_error", "fpg_abi_version",
    "fpg_ctx_create", "fpg_ctx_destroy", "fpg_ctx_stream", "fpg_ctx_synchronize", "fpg_ctx_kernel_launches",
    "fpg_device_alloc", "fpg_device_free", "fpg_memcpy", "fpg_memset", "fpg_host_alloc", "fpg_host_free",
    "fpg_particles_create", "fpg_particles_destroy", "fpg_particles_capacity", "fpg_particles_dispatch_count",
    "fpg_particles_set_dispatch_count", "fpg_particles_upload", "fpg_particles_upload_slots",
    "fpg_particles_download", "fpg_particles_field", "fpg_particles_copy_field",
    "fpg_step_tuning_candidates", "fpg_step_autotune", "fpg_step_set_tuning", "fpg_step_get_tuning",
    "fpg_met_create", "fpg_met_destroy", "fpg_met_upload_frame", "fpg_met_upload_frame_device",
    "fpg_met_upload_bracket_device",
    "fpg_met_set_level_heights",
    "fpg_pbl_create", "fpg_pbl_destroy", "fpg_pbl_upload", "fpg_pbl_download",
    "fpg_surface_create", "fpg_surface_destroy", "fpg_surface_upload", "fpg_pbl_diagnostics",
    "fpg_cellfield_create", "fpg_cellfield_destroy", "fpg_cellfield_upload", "fpg_cellfield_from_precipitation",
    "fpg_step_params_default", "fpg_step", "fpg_advect_dual_wind", "fpg_langevin_fused",
    "fpg_dry_deposition", "fpg_wet_deposition",
    "fpg_grid_create", "fpg_grid_destroy", "fpg_grid_accumulate", "fpg_grid_cell_indices", "fpg_grid_download",
    "fpg_grid_counts_device", "fpg_grid_mass_device", "fpg_grid_download_async",
    "fpg_compaction_create", "fpg_compaction_destroy", "fpg_compact",
    "fpg_philox_uniforms",
    "fpg_compaction_indices_static",
    "fpg_sorter_create", "fpg_sorter_destroy", "fpg_sort_by_cell",
    "fpg_dispatch_hanna_params", "fpg_langevin_with_hanna", "fpg_cbl_sample", "fpg_cbl_sample_philox",
    "fpg_convection_build_chain", "fpg_convection_level_index", "fpg_convection_apply_profile",
    "fpg_convection_create", "fpg_convection_destroy", "fpg_convection_set_matrix", "fpg_convection_heights",
    "fpg_convective_mixing",
]

# Every symbol include/fpg_driver.h declares.
EXPORTED_DRIVER = [
    "fpg_forward_config_default", "fpg_forward_create", "fpg_forward_destroy", "fpg_forward_has_remaining_steps",
    "fpg_forward_current_time", "fpg_forward_run_timestep", "fpg_forward_finalize", "fpg_forward_particles",
    "fpg_forward_accumulate_grid", "fpg_parse_timestamp",
    "fpg_forward_met_ring", "fpg_forward_prefetch_frame", "fpg_forward_met_ring_stats",
    "fpg_forward_set_profiling", "fpg_forward_last_timing", "fpg_forward_set_validation_mode",
    "fpg_backward_config_default", "fpg_backward_create", "fpg_backward_destroy", "fpg_backward_has_remaining_steps",
    "fpg_backward_current_time", "fpg_backward_run_timestep", "fpg_backward_particles",
    "fpg_backward_set_validation_mode",
    "fpg_batch_create", "fpg_batch_destroy", "fpg_batch_upload_frame", "fpg_batch_run", "fpg_batch_run_sequential",
    "fpg_batch_steps_done", "fpg_batch_scenario_slots", "fpg_batch_particles", "fpg_batch_download_grids",
    "fpg_batch_errors", "fpg_batch_tuning_candidates", "fpg_batch_autotune", "fpg_batch_set_tuning",
    "fpg_batch_get_tuning",
]

# Every symbol include/fpg_adjoint.h declares.
EXPORTED_ADJOINT = [
    "fpg_inverse_create", "fpg_inverse_destroy", "fpg_inverse_upload_frame", "fpg_inverse_set_sources",
    "fpg_inverse_set_wind_bias", "fpg_inverse_forward", "fpg_inverse_backward", "fpg_inverse_batch",
    "fpg_inverse_device_bytes",
]
