"""ctypes binding of libfvb200.so (the C ABI declared in include/fv_b200.h).

Loading never falls back to anything: if the shared library is missing the
import raises, and every device entry point reports CUDA errors as FvError.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfvb200.so"

FV_STATUS = {
    0: "FV_OK", 1: "FV_ERR_ALLOC", 2: "FV_ERR_INVALID", 3: "FV_ERR_SINGULAR_PIVOT", 4: "FV_ERR_BREAKDOWN",
    5: "FV_ERR_TIMEOUT", 6: "FV_ERR_NOT_SYMMETRIC", 7: "FV_ERR_CUDA", 8: "FV_ERR_UNSUPPORTED", 9: "FV_ERR_COMM",
}
FV_OK, FV_ERR_ALLOC, FV_ERR_INVALID, FV_ERR_SINGULAR_PIVOT, FV_ERR_BREAKDOWN = 0, 1, 2, 3, 4
FV_ERR_TIMEOUT, FV_ERR_NOT_SYMMETRIC, FV_ERR_CUDA, FV_ERR_UNSUPPORTED, FV_ERR_COMM = 5, 6, 7, 8, 9


class FvError(RuntimeError):
    """A status other than FV_OK; the reference panics in the same situations."""

    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = FV_STATUS.get(status, f"status {status}")
        detail = ""
        try:
            detail = lib().fv_last_error().decode()
        except Exception:  # pragma: no cover - best effort
            pass
        super().__init__(f"{what}: {name}" + (f" ({detail})" if detail and status == FV_ERR_CUDA else ""))


P = C.POINTER
dp, ip, i64 = P(C.c_double), P(C.c_int32), C.c_int64


class HostMesh_(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("n_nodes", i64), ("n_faces", i64), ("n_cells", i64), ("n_boundary_faces", i64),
        ("nodes", dp), ("face_node_ptr", ip), ("face_nodes", ip), ("face_patch", ip),
        ("cell_face_ptr", ip), ("cell_faces", ip), ("face_owner", ip), ("face_neighbor", ip),
        ("face_area", dp), ("face_normal", dp), ("face_center", dp), ("cell_center", dp), ("cell_volume", dp),
    ]


class MeshDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("n_cells", i64), ("n_faces", i64), ("n_boundary_faces", i64),
        ("face_owner", ip), ("face_neighbor", ip), ("face_area", dp), ("face_center", dp),
        ("cell_center", dp), ("cell_volume", dp), ("face_normal", dp), ("cell_face_ptr", ip), ("cell_faces", ip),
    ]


class TermsDesc(C.Structure):
    _fields_ = [
        ("laplacian_coef", C.c_double), ("convection_coef", C.c_double), ("source_coef", C.c_double),
        ("diffusivity", C.c_void_p), ("flux", C.c_void_p), ("source", C.c_void_p),
        ("scheme", C.c_int32), ("corrector_reduction", C.c_double), ("gradients", C.c_void_p),
        ("time_coef", C.c_double), ("time_scheme", C.c_int32), ("dt", C.c_double), ("dt_2", C.c_double),
        ("previous", C.c_void_p), ("previous_2", C.c_void_p), ("density", C.c_void_p),
        ("density_previous", C.c_void_p), ("density_previous_2", C.c_void_p),
        ("linear_source_coef", C.c_double), ("linear_source", C.c_void_p),
        ("divergence_coef", C.c_double), ("divergence_flux", C.c_void_p),
    ]


class BcDesc(C.Structure):
    _fields_ = [("bndi", C.c_void_p), ("bnde", C.c_void_p)]


class SolverOptions(C.Structure):
    _fields_ = [("relative_tolerance", C.c_double), ("absolute_tolerance", C.c_double),
                ("max_iterations", i64)]


class SolverInfo(C.Structure):
    _fields_ = [
        ("iterations", i64), ("initial_residual", C.c_double), ("final_residual", C.c_double),
        ("status", C.c_int32), ("restarts", C.c_int32), ("history", dp), ("history_cap", i64),
        ("history_len", i64), ("device_ms", C.c_double),
    ]


class BatchOptions(C.Structure):
    _fields_ = [("precision", C.c_int32), ("relative_tolerance", C.c_double), ("absolute_tolerance", C.c_double),
                ("max_iterations", i64), ("inner_relative_tolerance", C.c_double), ("outer_tolerance", C.c_double),
                ("max_outer", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("launched_iterations", i64), ("iterations", P(i64)),
                ("outer_steps", ip), ("final_residual", dp), ("status", ip), ("fp64_fallback", ip)]


# fv_comm: the collect / reduce_add callbacks of a distributed solve
COLLECT_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)
REDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)


class FvComm(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("collect", COLLECT_FN), ("reduce_add", REDUCE_FN)]


vp = C.c_void_p
class OrderInfo(C.Structure):
    """fv_order_info: the box-colour ordering's grid, colours and levels."""
    _fields_ = [("n_boxes", C.c_int64), ("boxes_per_axis", C.c_int32 * 3), ("n_colours", C.c_int32),
                ("n_levels", C.c_int32)]


_SIGS = {
    # host mesh
    "fv_host_mesh_from_elements": [C.c_int32, i64, dp, i64, ip, ip, ip, i64, ip, ip, ip, P(P(HostMesh_))],
    "fv_host_mesh_read_su2": [C.c_char_p, C.c_int32, P(P(HostMesh_))],
    "fv_host_mesh_generate_square": [C.c_int32, C.c_double, C.c_uint64, P(P(HostMesh_))],
    "fv_host_mesh_generate_cube": [C.c_int32, C.c_double, C.c_uint64, P(P(HostMesh_))],
    "fv_host_fields_generate": [P(HostMesh_), C.c_uint64, C.c_double, C.c_double, dp, C.c_double, C.c_int32,
                                dp, dp, dp],
    # device objects
    "fv_mesh_upload": [P(MeshDesc), vp, P(vp)],
    "fv_mesh_build_elements": [C.c_int32, i64, dp, i64, ip, ip, ip, i64, ip, ip, ip, vp, P(vp), P(P(HostMesh_))],
    "fv_mesh_build_su2": [C.c_char_p, C.c_int32, vp, P(vp), P(P(HostMesh_))],
    "fv_mesh_build_msh": [C.c_char_p, C.c_int32, vp, P(vp), P(P(HostMesh_))],
    "fv_mesh_concat": [P(vp), C.c_int32, vp, P(vp)],
    "fv_mesh_build_faces": [C.c_int32, i64, dp, i64, ip, ip, ip, i64, ip, ip, vp, P(vp), P(P(HostMesh_))],
    "fv_host_mesh_from_faces": [C.c_int32, i64, dp, i64, ip, ip, ip, i64, ip, ip, P(P(HostMesh_))],
    "fv_host_mesh_read_msh": [C.c_char_p, C.c_int32, P(P(HostMesh_))],
    "fv_host_mesh_write_msh": [P(HostMesh_), C.c_char_p, P(C.c_char_p), C.c_int32],
    "fv_mesh_build_square": [C.c_int32, C.c_double, C.c_uint64, vp, P(vp), P(P(HostMesh_))],
    "fv_mesh_build_cube": [C.c_int32, C.c_double, C.c_uint64, vp, P(vp), P(P(HostMesh_))],
    "fv_mesh_destroy": [vp],
    "fv_compute_gradients": [vp, vp, P(BcDesc), vp, vp],
    "fv_assemble": [vp, P(TermsDesc), P(BcDesc), P(vp), vp, vp],
    "fv_assemble_host": [vp, P(TermsDesc), P(BcDesc), P(vp), dp, vp],
    "fv_csr_create_host": [i64, i64, ip, ip, dp, vp, P(vp)],
    "fv_csr_info": [vp, P(i64), P(i64), P(i64)],
    "fv_csr_download": [vp, ip, ip, dp, vp],
    "fv_csr_destroy": [vp],
    "fv_spmv": [vp, vp, vp, vp],
    "fv_spmv_host": [vp, dp, dp, vp],
    "fv_ic0_factor": [vp, vp, P(vp)],
    "fv_ilu0_factor": [vp, vp, P(vp)],
    "fv_diag_factor": [vp, vp, P(vp)],
    "fv_vec_dot": [i64, vp, vp, vp, P(C.c_double)],
    "fv_vec_sum": [i64, vp, vp, P(C.c_double)],
    "fv_vec_update": [i64, vp, vp, C.c_double, C.c_int32, vp],
    "fv_ic_factor": [vp, C.c_int32, vp, P(vp)],
    "fv_ilu_factor": [vp, C.c_int32, vp, P(vp)],
    "fv_precond_refactor": [vp, vp],
    "fv_precond_apply": [vp, vp, vp, vp],
    "fv_precond_apply_host": [vp, dp, dp, vp],
    "fv_precond_export": [vp, P(i64), ip, ip, dp, ip, vp],
    "fv_precond_levels": [vp, ip, ip, ip, ip, vp],
    "fv_precond_destroy": [vp],
    "fv_precond_schedule": [vp, C.c_int32, P(C.c_int32), dp],
    "fv_tile_plan_host": [i64, C.c_int32, dp, ip, ip, C.c_int32, P(i64), ip, ip, ip, ip, dp],
    "fv_fill_pattern_host": [C.c_int32, C.c_int32, i64, ip, ip, P(i64), ip, ip, ip, P(C.c_uint8)],
    "fv_cg": [vp, vp, vp, vp, SolverOptions, P(SolverInfo), vp],
    "fv_bicgstab": [vp, vp, vp, vp, SolverOptions, P(SolverInfo), vp],
    "fv_cg_host": [vp, vp, dp, dp, SolverOptions, P(SolverInfo), vp],
    "fv_bicgstab_host": [vp, vp, dp, dp, SolverOptions, P(SolverInfo), vp],
    "fv_cg_noalloc": [vp, vp, vp, vp, SolverOptions, P(SolverInfo), vp],
    "fv_ic0_factor_perm": [vp, ip, vp, P(vp)],
    "fv_ilu0_factor_perm": [vp, ip, vp, P(vp)],
    "fv_precond_perm": [vp, ip, vp],
    "fv_precond_set_grid": [vp, C.c_int32, C.c_int32],
    "fv_order_boxes_host": [i64, C.c_int32, dp, i64, dp, dp, ip, ip, C.c_int32, ip, P(OrderInfo)],
    "fv_order_boxes_batch_host": [C.c_int32, P(i64), C.c_int32, dp, i64, dp, dp, ip, ip, C.c_int32, ip,
                                  P(OrderInfo)],
    "fv_order_boxes": [vp, C.c_int32, P(i64), C.c_int32, ip, P(OrderInfo), vp],
    "fv_order_boxes_levels": [vp, C.c_int32, ip, ip, P(OrderInfo), vp],
    "fv_csr_permute": [vp, ip, vp, P(vp)],
    "fv_csr_permute_values": [vp, vp],
    "fv_vec_permute": [vp, vp, vp, C.c_int32, vp],
    "fv_order_boxes_host_levels": [i64, C.c_int32, dp, i64, dp, dp, ip, ip, C.c_int32, ip, ip, P(OrderInfo)],
    "fv_batch_create": [vp, C.c_int32, P(i64), C.c_int32, vp, P(vp)],
    "fv_batch_cg": [vp, vp, vp, vp, P(BatchOptions), P(BatchInfo), vp],
    "fv_batch_bicgstab": [vp, vp, vp, vp, P(BatchOptions), P(BatchInfo), vp],
    "fv_batch_destroy": [vp],
    "fv_batch_begin": [vp, vp, C.c_int32, vp, vp, P(BatchOptions), vp, P(C.c_int32), vp],
    "fv_batch_advance": [vp, C.c_int64, P(C.c_int32), P(C.c_int32), vp],
    "fv_batch_report": [vp, P(BatchInfo)],
    "fv_csr_square_block": [vp, vp, P(vp)],
    "fv_dist_create": [vp, i64, ip, i64, P(FvComm), P(vp)],
    "fv_dist_destroy": [vp],
    "fv_dist_spmv": [vp, vp, vp, vp],
    "fv_dist_dot": [vp, vp, vp, dp, vp],
    "fv_dist_cg": [vp, vp, vp, vp, SolverOptions, P(SolverInfo), vp],
    "fv_dist_bicgstab": [vp, vp, vp, vp, SolverOptions, P(SolverInfo), vp],
}

_lib = None
_exiting = False


def _mark_exit():
    global _exiting
    _exiting = True


# Python runs atexit handlers before it tears modules down.  From then on the
# finalizers of device objects skip their native frees: the process is ending
# (the driver reclaims everything), and native calls from finalizers that run
# during interpreter teardown, after other libraries' own teardown, are not safe.
atexit.register(_mark_exit)


def exiting() -> bool:
    return _exiting


def lib() -> C.CDLL:
    """Load libfvb200.so (built in-tree by build.py).  Raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() (or fvb200/build.py)")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.fv_host_mesh_free.argtypes = [P(HostMesh_)]
        L.fv_host_mesh_free.restype = None
        L.fv_status_string.argtypes = [C.c_int]
        L.fv_status_string.restype = C.c_char_p
        L.fv_last_error.argtypes = []
        L.fv_last_error.restype = C.c_char_p
        L.fv_launch_count.argtypes = []
        L.fv_launch_count.restype = C.c_uint64
        _lib = L
    return _lib


def check(status: int, what: str) -> None:
    if status != FV_OK:
        raise FvError(status, what)


def exported_symbols() -> list[str]:
    return list(_SIGS) + ["fv_host_mesh_free", "fv_status_string", "fv_last_error", "fv_launch_count"]
