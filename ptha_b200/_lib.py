"""ctypes binding of libswalsgpu.so (include/swals_gpu.h).

The shared library is the product; this module only declares its C ABI.  It
fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libswalsgpu.so")

SWALS_OK = 0
ERRORS = {
    1: "SWALS_ERR_INVALID_ARGUMENT", 2: "SWALS_ERR_UNKNOWN_METHOD", 3: "SWALS_ERR_UNSUPPORTED",
    4: "SWALS_ERR_CUDA", 5: "SWALS_ERR_NONFINITE", 6: "SWALS_ERR_UNSUPPORTED_CALLBACK",
    7: "SWALS_ERR_TIMESTEP_REQUIRED", 8: "SWALS_ERR_OUT_OF_MEMORY", 9: "SWALS_ERR_NO_DEVICE",
    10: "SWALS_ERR_CAPACITY",
}
BC_NONE, BC_TRANSMISSIVE, BC_STAGE_TRANSMISSIVE_NORMAL_MOMENTUM, BC_FLATHER = 0, 1, 2, 3
BF_NONE, BF_SOLITARY_WEST_WALLS = 0, 1
FRICTION_MANNING, FRICTION_CHEZY = 0, 1

# Every symbol include/swals_gpu.h declares.
EXPORTED = [
    "swals_gpu_desc_init", "swals_gpu_domain_create", "swals_gpu_domain_destroy",
    "swals_gpu_upload_U", "swals_gpu_download_U", "swals_gpu_upload_var", "swals_gpu_download_var",
    "swals_gpu_upload_manning_squared", "swals_gpu_get_metrics", "swals_gpu_upload_metrics",
    "swals_gpu_evolve_one_step", "swals_gpu_evolve_steps", "swals_gpu_get_state", "swals_gpu_set_time",
    "swals_gpu_synchronize", "swals_gpu_download_max_stage", "swals_gpu_linear_timestep_max",
    "swals_gpu_nonlinear_stationary_timestep_max", "swals_gpu_stationary_timestep_max",
    "swals_gpu_volume_interior", "swals_gpu_gauges_setup", "swals_gpu_gauges_site_index",
    "swals_gpu_gauges_read", "swals_gpu_gauges_reset", "swals_gpu_timers_enable", "swals_gpu_timers_read",
    "swals_gpu_stream", "swals_gpu_device_planes", "swals_gpu_last_error", "swals_gpu_version",
    "swals_gpu_launch_count",
    "swals_gpu_batch_create", "swals_gpu_batch_destroy", "swals_gpu_batch_upload_U", "swals_gpu_batch_download_U",
    "swals_gpu_batch_download_max_stage", "swals_gpu_batch_device_state", "swals_gpu_batch_gauges_setup",
    "swals_gpu_batch_gauges_read", "swals_gpu_batch_evolve", "swals_gpu_batch_time", "swals_gpu_batch_tune",
    "swals_gpu_batch_set_tile_config", "swals_gpu_batch_tile_config_count", "swals_gpu_adjoint_linear", "swals_gpu_misfit_gradient_linear",
    "swals_gpu_volume_interior_noalloc",
    "swals_gpu_md_create", "swals_gpu_md_destroy", "swals_gpu_md_evolve_one_step", "swals_gpu_md_send_halos",
    "swals_gpu_md_recv_halos", "swals_gpu_md_flux_correction", "swals_gpu_md_buffer_size",
    "swals_gpu_md_download_buffer", "swals_gpu_md_download_flux", "swals_gpu_md_time", "swals_gpu_md_synchronize",
    "swals_gpu_md_launch_count", "swals_gpu_md_capture_graph", "swals_gpu_md_replay",
    "swals_gpu_md_group_create", "swals_gpu_md_group_replay", "swals_gpu_md_group_stream",
    "swals_gpu_md_group_destroy",
    "swals_gpu_set_priority_mask", "swals_gpu_domain_statistics", "swals_gpu_volume_in_priority_domain",
    "swals_gpu_forcing_patch_add", "swals_gpu_forcing_clear", "swals_gpu_apply_forcing",
    "swals_gpu_set_eddy_viscosity", "swals_gpu_set_static_before_time", "swals_gpu_set_max_U_update_frequency",
    "swals_gpu_set_max_U_variables", "swals_gpu_download_max_U",
    "swals_md_build_metadata", "swals_md_metadata_exchanges", "swals_md_metadata_priority",
    "swals_md_metadata_recv_boxes", "swals_md_metadata_free",
    "swals_gpu_stage_grids_real4", "swals_gpu_gauges_read_real4",
]
TIMER_NAMES = ["cfl", "fv_stage1", "boundary1", "fv_stage2", "boundary2", "finalize", "leapfrog_edge",
               "leapfrog_step", "gauges", "max_stage"]


class SwalsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class DomainDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32 * 2), ("lw", ctypes.c_double * 2), ("lower_left", ctypes.c_double * 2),
        ("timestepping_method", ctypes.c_char * 64),
        ("cfl", ctypes.c_double), ("theta", ctypes.c_double), ("msl_linear", ctypes.c_double),
        ("linear_friction_coeff", ctypes.c_double), ("maximum_timestep", ctypes.c_double),
        ("linear_solver_is_truely_linear", ctypes.c_int32), ("friction_type", ctypes.c_int32),
        ("spherical", ctypes.c_int32), ("coriolis", ctypes.c_int32), ("nofriction", ctypes.c_int32),
        ("real_bytes", ctypes.c_int32),
        ("xL", ctypes.c_int32), ("xU", ctypes.c_int32), ("yL", ctypes.c_int32), ("yU", ctypes.c_int32),
        ("boundary_exterior", ctypes.c_int32 * 4), ("boundary_kind", ctypes.c_int32),
        ("boundary_function_kind", ctypes.c_int32), ("boundary_function_params", ctypes.c_double * 8),
        ("record_max_stage", ctypes.c_int32), ("exterior_cells_width", ctypes.c_int32),
        ("has_host_boundary_subroutine", ctypes.c_int32), ("has_host_forcing_subroutine", ctypes.c_int32),
        ("device", ctypes.c_int32), ("compute_fluxes_inner_method", ctypes.c_char * 64),
    ]


class NestExchange(ctypes.Structure):
    _fields_ = [("sender", ctypes.c_int32), ("receiver", ctypes.c_int32),
                ("send_box", ctypes.c_int32 * 4), ("recv_box", ctypes.c_int32 * 4)]


class DomainState(ctypes.Structure):
    _fields_ = [
        ("time", ctypes.c_double), ("max_dt", ctypes.c_double), ("dt_last_update", ctypes.c_double),
        ("evolve_step_dt", ctypes.c_double), ("nsteps_advanced", ctypes.c_int64),
        ("negative_depth_fix_counter", ctypes.c_int64), ("boundary_flux_store", ctypes.c_double * 4),
        ("boundary_flux_evolve_integral", ctypes.c_double), ("boundary_flux_time_integral", ctypes.c_double),
    ]


_lib = None


def lib():
    """Load libswalsgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m ptha_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    sig = {
        "swals_gpu_desc_init": [ctypes.POINTER(DomainDesc)],
        "swals_gpu_domain_create": [ctypes.POINTER(DomainDesc), ctypes.POINTER(vp)],
        "swals_gpu_domain_destroy": [vp],
        "swals_gpu_upload_U": [vp, vp], "swals_gpu_download_U": [vp, vp],
        "swals_gpu_upload_var": [vp, i32, vp], "swals_gpu_download_var": [vp, i32, vp],
        "swals_gpu_upload_manning_squared": [vp, vp],
        "swals_gpu_get_metrics": [vp] + [vp] * 8,
        "swals_gpu_upload_metrics": [vp] + [vp] * 6,
        "swals_gpu_evolve_one_step": [vp, dbl, i32],
        "swals_gpu_evolve_steps": [vp, i32, dbl, i32],
        "swals_gpu_get_state": [vp, ctypes.POINTER(DomainState)],
        "swals_gpu_set_time": [vp, dbl], "swals_gpu_synchronize": [vp],
        "swals_gpu_download_max_stage": [vp, vp],
        "swals_gpu_linear_timestep_max": [vp, ctypes.POINTER(dbl)],
        "swals_gpu_nonlinear_stationary_timestep_max": [vp, ctypes.POINTER(dbl)],
        "swals_gpu_stationary_timestep_max": [vp, ctypes.POINTER(dbl)],
        "swals_gpu_volume_interior": [vp, ctypes.POINTER(dbl)],
        "swals_gpu_gauges_setup": [vp, vp, i32, i32],
        "swals_gpu_gauges_site_index": [vp, vp],
        "swals_gpu_gauges_read": [vp, vp, i32, ctypes.POINTER(i32)],
        "swals_gpu_gauges_reset": [vp],
        "swals_gpu_timers_enable": [vp, i32],
        "swals_gpu_timers_read": [vp, vp, i32, ctypes.POINTER(i32)],
        "swals_gpu_stream": [vp, ctypes.POINTER(vp)],
        "swals_gpu_device_planes": [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                    ctypes.POINTER(vp), ctypes.POINTER(i64)],
        "swals_gpu_last_error": [ctypes.c_char_p, ctypes.c_size_t],
        "swals_gpu_launch_count": [vp, ctypes.POINTER(i64)],
        "swals_gpu_batch_create": [vp, i32, i32, ctypes.POINTER(vp)],
        "swals_gpu_batch_destroy": [vp],
        "swals_gpu_batch_upload_U": [vp, i32, i32, vp],
        "swals_gpu_batch_download_U": [vp, i32, i32, vp],
        "swals_gpu_batch_download_max_stage": [vp, i32, i32, vp],
        "swals_gpu_batch_device_state": [vp, ctypes.POINTER(vp), ctypes.POINTER(i64), ctypes.POINTER(i64),
                                         ctypes.POINTER(i64)],
        "swals_gpu_batch_gauges_setup": [vp, vp, i32, i32],
        "swals_gpu_batch_gauges_read": [vp, vp, i32, ctypes.POINTER(i32)],
        "swals_gpu_batch_evolve": [vp, i32, dbl],
        "swals_gpu_batch_time": [vp, ctypes.POINTER(dbl), ctypes.POINTER(i64)],
        "swals_gpu_batch_tune": [vp, ctypes.POINTER(i32), ctypes.POINTER(dbl)],
        "swals_gpu_batch_set_tile_config": [vp, i32],
        "swals_gpu_batch_tile_config_count": [ctypes.POINTER(i32)],
        "swals_gpu_adjoint_linear": [vp, i32, dbl, vp, vp, vp],
        "swals_gpu_misfit_gradient_linear": [vp, i32, dbl, vp, i32, ctypes.POINTER(dbl), vp],
        "swals_gpu_volume_interior_noalloc": [vp, vp, vp, i32, i32, i64, i32, i32, vp, vp],
        "swals_gpu_md_create": [vp, i32, vp, vp, vp, i32, vp, i32, i32, ctypes.POINTER(vp)],
        "swals_gpu_md_destroy": [vp], "swals_gpu_md_evolve_one_step": [vp, dbl],
        "swals_gpu_md_send_halos": [vp], "swals_gpu_md_recv_halos": [vp], "swals_gpu_md_flux_correction": [vp],
        "swals_gpu_md_buffer_size": [vp, i32, ctypes.POINTER(i64)],
        "swals_gpu_md_download_buffer": [vp, i32, vp, i64],
        "swals_gpu_md_download_flux": [vp, i32, i32, vp, i64],
        "swals_gpu_md_time": [vp, ctypes.POINTER(dbl)], "swals_gpu_md_synchronize": [vp],
        "swals_gpu_md_launch_count": [vp, ctypes.POINTER(i64)],
        "swals_gpu_md_capture_graph": [vp, i32, dbl], "swals_gpu_md_replay": [vp, i32],
        "swals_gpu_md_group_create": [vp, i32, i32, dbl, ctypes.POINTER(vp)],
        "swals_gpu_md_group_replay": [vp, i32], "swals_gpu_md_group_stream": [vp, ctypes.POINTER(vp)],
        "swals_gpu_md_group_destroy": [vp],
        "swals_gpu_set_priority_mask": [vp, vp], "swals_gpu_domain_statistics": [vp, vp],
        "swals_gpu_volume_in_priority_domain": [vp, ctypes.POINTER(dbl)],
        "swals_gpu_forcing_patch_add": [vp, i32, i32, i32, i32, i32, i32, dbl, dbl, vp, ctypes.POINTER(i32)],
        "swals_gpu_forcing_clear": [vp], "swals_gpu_apply_forcing": [vp, dbl],
        "swals_gpu_set_eddy_viscosity": [vp, i32, dbl, dbl],
        "swals_gpu_set_static_before_time": [vp, dbl], "swals_gpu_set_max_U_update_frequency": [vp, i32],
        "swals_gpu_set_max_U_variables": [vp, i32, i32, dbl], "swals_gpu_download_max_U": [vp, i32, vp],
        "swals_md_build_metadata": [vp, i32, i32, i32, vp, vp, ctypes.POINTER(vp)],
        "swals_md_metadata_exchanges": [vp, vp, i32, ctypes.POINTER(i32)],
        "swals_md_metadata_priority": [vp, i32, vp, vp],
        "swals_md_metadata_recv_boxes": [vp, i32, vp, i32, ctypes.POINTER(i32)],
        "swals_gpu_stage_grids_real4": [vp, i32, i32, vp, i64, vp],
        "swals_gpu_gauges_read_real4": [vp, vp, i32, ctypes.POINTER(i32)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.swals_md_metadata_free.argtypes = [vp]
    L.swals_md_metadata_free.restype = None
    L.swals_gpu_version.restype = ctypes.c_char_p
    L.swals_gpu_version.argtypes = []
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().swals_gpu_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != SWALS_OK:
        raise SwalsError(rc, last_error())
