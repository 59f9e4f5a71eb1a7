"""ctypes binding of libfdtd_b200.so (include/fdtd_c.h).

There is no fallback: if the library cannot be loaded the import of the solver
fails with the reason.
"""
from __future__ import annotations

import ctypes as C
import os

from .scene import GaussianSourceDesc, GhostFace, Options, SceneDesc, ServerConfig, ServerStats, SolverInfo

HERE = os.path.dirname(os.path.abspath(__file__))
# FDTD_B200_LIB: load another build of the same library (same ABI), e.g. one with
# other compile-time tile shapes
LIB_PATH = os.environ.get("FDTD_B200_LIB") or os.path.join(HERE, "_lib", "libfdtd_b200.so")

# every symbol include/fdtd_c.h declares
EXPORTS = [
    "fdtd_abi_version", "fdtd_last_error", "fdtd_device_count", "fdtd_debug_inject_failure", "fdtd_gaussian_source_defaults",
    "fdtd_solver_create", "fdtd_solver_destroy", "fdtd_release_cached_memory", "fdtd_solver_reset", "fdtd_solver_step",
    "fdtd_solver_step_device", "fdtd_solver_fetch_listeners", "fdtd_solver_info_get",
    "fdtd_solver_get_classification", "fdtd_solver_get_field", "fdtd_solver_synchronize",
    "fdtd_solver_stream", "fdtd_solver_last_error", "fdtd_solver_last_launch_count", "fdtd_solver_pml_state", "fdtd_solver_shell_staging",
    "fdtd_solver_overlapped_steps", "fdtd_solver_transfer_bytes", "fdtd_read_obj",
    "fdtd_read_kinematics", "fdtd_keyframe_pose", "fdtd_mesh_signed_distance",
    "fdtd_solver_prepare_graphs", "fdtd_solver_set_field", "fdtd_matrix_write", "fdtd_matrix_read",
    "fdtd_solver_save_snapshot", "fdtd_solver_load_snapshot", "fdtd_solver_save_config",
    "fdtd_solver_save_field_timestep", "fdtd_solver_boundary_info",
    "fdtd_solver_snapshot", "fdtd_solver_restore", "fdtd_scene_from_xml", "fdtd_scene_desc_get",
    "fdtd_scene_number_of_steps", "fdtd_scene_output_pattern", "fdtd_scene_free", "fdtd_audio_append",
    "fdtd_solver_time_stencil", "fdtd_solver_time_kernel", "fdtd_interior_step_noalloc",
    "fdtd_batch_create", "fdtd_batch_add", "fdtd_batch_step", "fdtd_batch_run", "fdtd_batch_member_info",
    "fdtd_batch_output", "fdtd_batch_release", "fdtd_batch_destroy", "fdtd_batch_stream",
    "fdtd_batch_last_launch_count", "fdtd_batch_device_bytes", "fdtd_scene_device_bytes", "fdtd_scene_info",
    "fdtd_server_create", "fdtd_server_submit", "fdtd_server_poll", "fdtd_server_wait", "fdtd_server_result",
    "fdtd_server_drain", "fdtd_server_stats_get", "fdtd_server_request_error", "fdtd_server_destroy",
    "fdtd_server_cancel", "fdtd_batch_member_snapshot", "fdtd_batch_add_snapshot",
    "fdtd_solver_fetch_cell", "fdtd_solver_sample_slice", "fdtd_solver_domain",
]

_lib = None


class FDTDError(RuntimeError):
    def __init__(self, status: int, msg: str):
        from .scene import STATUS
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def load(build_if_missing: bool = False):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from .build import build
            build()
        else:
            raise ImportError(f"{LIB_PATH} is missing: run `python -m acoustics_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    sig = {
        "fdtd_abi_version": ([], i32),
        "fdtd_last_error": ([], C.c_char_p),
        "fdtd_device_count": ([C.POINTER(i32)], i32),
        "fdtd_debug_inject_failure": ([i32, i32], i32),
        "fdtd_gaussian_source_defaults": ([C.POINTER(GaussianSourceDesc), dbl], i32),
        "fdtd_solver_create": ([C.POINTER(SceneDesc), C.POINTER(Options), C.POINTER(vp)], i32),
        "fdtd_solver_destroy": ([vp], i32),
        "fdtd_release_cached_memory": ([i32], None),
        "fdtd_solver_reset": ([vp, dbl], i32),
        "fdtd_solver_step": ([vp, i32, vp], i32),
        "fdtd_solver_step_device": ([vp, i32, vp], i32),
        "fdtd_solver_fetch_listeners": ([vp, vp], i32),
        "fdtd_solver_info_get": ([vp, C.POINTER(SolverInfo)], i32),
        "fdtd_solver_get_classification": ([vp, vp, vp, C.POINTER(i64)], i32),
        "fdtd_solver_get_field": ([vp, i32, vp, i64], i32),
        "fdtd_solver_synchronize": ([vp], i32),
        "fdtd_solver_stream": ([vp], vp),
        "fdtd_solver_last_error": ([vp], C.c_char_p),
        "fdtd_solver_last_launch_count": ([vp], i64),
        "fdtd_solver_overlapped_steps": ([vp], i64),
        "fdtd_solver_transfer_bytes": ([vp, C.POINTER(i64), C.POINTER(i64)], i32),
        "fdtd_read_obj": ([C.c_char_p, dbl, C.POINTER(i32), C.POINTER(i32), vp, vp], i32),
        "fdtd_read_kinematics": ([C.c_char_p, C.POINTER(i32), vp, i64], i32),
        "fdtd_keyframe_pose": ([vp, dbl, vp, vp], i32),
        "fdtd_mesh_signed_distance": ([vp, i64, vp, vp], i32),
        "fdtd_solver_pml_state": ([vp], i32),
        "fdtd_solver_shell_staging": ([vp], i32),
        "fdtd_solver_prepare_graphs": ([vp], i32),
        "fdtd_solver_set_field": ([vp, i32, vp, i64], i32),
        "fdtd_solver_fetch_cell": ([vp, i64, vp], i32),
        "fdtd_solver_domain": ([vp, vp, vp], i32),
        "fdtd_solver_sample_slice": ([vp, i32, dbl, vp, i64, C.POINTER(i64)], i32),
        "fdtd_matrix_write": ([C.c_char_p, i32, i32, vp], i32),
        "fdtd_matrix_read": ([C.c_char_p, C.POINTER(i32), C.POINTER(i32), vp, i64], i32),
        "fdtd_solver_save_snapshot": ([vp, C.c_char_p, C.c_char_p], i32),
        "fdtd_solver_load_snapshot": ([vp, C.c_char_p, C.c_char_p], i32),
        "fdtd_solver_save_config": ([vp, C.c_char_p], i32),
        "fdtd_solver_save_field_timestep": ([vp, i32, C.c_char_p], i32),
        "fdtd_solver_boundary_info": ([vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(i32)], i32),
        "fdtd_solver_snapshot": ([vp, vp, C.POINTER(i64)], i32),
        "fdtd_solver_restore": ([vp, vp, i64], i32),
        "fdtd_scene_from_xml": ([C.c_char_p, C.POINTER(vp)], i32),
        "fdtd_scene_desc_get": ([vp], C.POINTER(SceneDesc)),
        "fdtd_scene_number_of_steps": ([vp], i32),
        "fdtd_scene_output_pattern": ([vp], C.c_char_p),
        "fdtd_scene_free": ([vp], None),
        "fdtd_audio_append": ([C.c_char_p, vp, i64], i32),
        "fdtd_solver_time_stencil": ([vp, i32, C.POINTER(C.c_float)], i32),
        "fdtd_solver_time_kernel": ([vp, i32, i32, C.POINTER(C.c_float)], i32),
        "fdtd_interior_step_noalloc": ([vp, vp, vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), dbl, dbl, vp],
                                       i32),
        "fdtd_batch_create": ([i32, C.POINTER(SceneDesc), C.POINTER(i32), C.POINTER(Options), C.POINTER(vp)], i32),
        "fdtd_batch_add": ([vp, C.POINTER(SceneDesc), i32, C.POINTER(i32)], i32),
        "fdtd_batch_step": ([vp, i32, C.POINTER(i32)], i32),
        "fdtd_batch_run": ([vp], i32),
        "fdtd_batch_member_info": ([vp, i32, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32), C.POINTER(i32)], i32),
        "fdtd_batch_output": ([vp, i32, vp, i64], i32),
        "fdtd_batch_release": ([vp, i32], i32),
        "fdtd_batch_destroy": ([vp], i32),
        "fdtd_batch_stream": ([vp], vp),
        "fdtd_batch_last_launch_count": ([vp], i64),
        "fdtd_batch_device_bytes": ([vp], i64),
        "fdtd_scene_device_bytes": ([C.POINTER(SceneDesc), C.POINTER(Options)], i64),
        "fdtd_scene_info": ([C.POINTER(SceneDesc), C.POINTER(Options), C.POINTER(SolverInfo)], i32),
        "fdtd_server_create": ([C.POINTER(Options), C.POINTER(ServerConfig), C.POINTER(vp)], i32),
        "fdtd_server_submit": ([vp, C.POINTER(SceneDesc), i32, C.POINTER(i64)], i32),
        "fdtd_server_poll": ([vp, i64, C.POINTER(i32), C.POINTER(i64), C.POINTER(i32)], i32),
        "fdtd_server_wait": ([vp, i64, dbl], i32),
        "fdtd_server_result": ([vp, i64, vp, i64, C.POINTER(i64), C.POINTER(i32), C.POINTER(dbl)], i32),
        "fdtd_server_drain": ([vp, dbl], i32),
        "fdtd_server_stats_get": ([vp, C.POINTER(ServerStats)], i32),
        "fdtd_server_request_error": ([vp, i64], C.c_char_p),
        "fdtd_server_destroy": ([vp], i32),
        "fdtd_server_cancel": ([vp, i64], i32),
        "fdtd_batch_member_snapshot": ([vp, i32, vp, C.POINTER(i64)], i32),
        "fdtd_batch_add_snapshot": ([vp, C.POINTER(SceneDesc), i32, vp, i64, vp, i64, C.POINTER(i32)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(status: int, handle=None) -> int:
    """Raise FDTDError for negative status codes; return the status otherwise."""
    if status < 0:
        L = load()
        msg = L.fdtd_solver_last_error(handle) if handle else L.fdtd_last_error()
        raise FDTDError(status, (msg or b"").decode(errors="replace"))
    return status
