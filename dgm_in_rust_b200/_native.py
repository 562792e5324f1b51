"""ctypes binding of the C ABI in include/dgm_b200.h (libdgm_b200.so, built in-tree).

There is no CPU fallback: if the shared library is missing or no CUDA device is usable, the
calls raise :class:`DgmError`.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["DgmError", "lib", "library_path", "MeshDesc", "TablesDesc", "Params", "SlotCapacity", "STATUS"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libdgm_b200.so"

STATUS = {
    0: "ok",
    1: "Negative density found in HLLC!",
    2: "Negative pressure found in HLLC!",
    3: "Non-finite value",
    4: "Invalid number of boundary neighbours!",
    5: "Device memory allocation failed",
    6: "Device wait timed out",
    7: "Invalid argument",
    9: "CUDA runtime error",
    10: "No usable CUDA device",
    11: "Work still in flight",
    12: "Limiter worklist overflow",
}
DGM_NOT_READY = 11


class DgmError(RuntimeError):
    """A non-OK status from the library; ``status`` holds the DGM_* code, ``where`` the edge or
    element the device flagged (the reference panics in these cases)."""

    def __init__(self, status: int, where: int = -1, what: str = ""):
        self.status = int(status)
        self.where = int(where)
        msg = STATUS.get(self.status, f"status {self.status}")
        if what:
            msg = f"{what}: {msg}"
        if where >= 0:
            msg += f" (at index {where})"
        super().__init__(msg)


def library_path() -> str:
    return os.path.join(_HERE, "_lib", LIB_NAME)


P_D = ctypes.POINTER(ctypes.c_double)
P_I64 = ctypes.POINTER(ctypes.c_int64)
P_I32 = ctypes.POINTER(ctypes.c_int32)


class MeshDesc(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int64),
        ("n_elements", ctypes.c_int64),
        ("n_edges", ctypes.c_int64),
        ("n_patches", ctypes.c_int64),
        ("vertex_xy", P_D),
        ("elem_vertices", P_I64),
        ("elem_edges", P_I64),
        ("elem_neighbours", P_I64),
        ("elem_jacob_det", P_D),
        ("elem_circumradius", P_D),
        ("elem_minimum_height", P_D),
        ("edge_elements", P_I64),
        ("edge_vertices", P_I64),
        ("edge_in_cell", P_I64),
        ("edge_jacob_det", P_D),
        ("edge_normal", P_D),
        ("edge_patch", P_I64),
        ("patch_type", P_I32),
        ("patch_quantity", P_D),
        ("n_internal_edges", ctypes.c_int64),
        ("internal_edges", P_I64),
        ("n_boundary_elements", ctypes.c_int64),
        ("boundary_elements", P_I64),
    ]


class TablesDesc(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int32),
        ("n_basis", ctypes.c_int32),
        ("n_cell_gp", ctypes.c_int32),
        ("n_edge_gp", ctypes.c_int32),
        ("n_deriv_keys", ctypes.c_int32),
        ("_pad", ctypes.c_int32),
        ("cell_weights", P_D),
        ("edge_weights", P_D),
        ("phi_cell", P_D),
        ("phi_edge", P_D),
        ("dphi_cell_ref", P_D),
        ("mass_diag", P_D),
    ]


class SlotCapacity(ctypes.Structure):
    _fields_ = [
        ("elements", ctypes.c_int64),
        ("internal_edges", ctypes.c_int64),
        ("boundary_edges", ctypes.c_int64),
        ("patches", ctypes.c_int64),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("hcr", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("final_time", ctypes.c_double),
        ("final_step", ctypes.c_int64),
        ("limiter", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("_reserved", ctypes.c_int32),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libdgm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise DgmError(10, what=f"{LIB_NAME} not built (run dgm_in_rust_b200.build.build())")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.dgm_create.argtypes = [ctypes.POINTER(MeshDesc), ctypes.POINTER(TablesDesc), ctypes.POINTER(Params), P_I32]
    L.dgm_create.restype = vp
    L.dgm_destroy.argtypes = [vp]
    L.dgm_destroy.restype = None
    L.dgm_compute_residuals.argtypes = [vp, P_D, P_D]
    L.dgm_apply_limiter.argtypes = [vp, P_D, P_I64]
    L.dgm_compute_time_step.argtypes = [vp, P_D, P_D]
    L.dgm_rk3.argtypes = [vp, P_D, P_D, ctypes.c_double]
    L.dgm_time_march.argtypes = [vp, P_D, P_D]
    L.dgm_get_clock.argtypes = [vp, P_D, P_I64]
    L.dgm_set_clock.argtypes = [vp, ctypes.c_double, ctypes.c_int64]
    L.dgm_set_limits.argtypes = [vp, ctypes.c_double, ctypes.c_int64]
    L.dgm_launch_phase.argtypes = [vp, ctypes.c_int32]
    L.dgm_phase_launches_per_step.argtypes = [vp, ctypes.c_int32]
    L.dgm_launches_per_step.argtypes = [vp]
    L.dgm_create_batch.argtypes = [ctypes.c_int32, ctypes.POINTER(MeshDesc), ctypes.POINTER(TablesDesc),
                                   ctypes.POINTER(Params), P_I32]
    L.dgm_create_batch.restype = vp
    L.dgm_instance_count.argtypes = [vp]
    L.dgm_create_batch_slots.argtypes = [ctypes.c_int32, ctypes.POINTER(MeshDesc), ctypes.POINTER(SlotCapacity),
                                         ctypes.POINTER(TablesDesc), ctypes.POINTER(Params), P_I32]
    L.dgm_create_batch_slots.restype = vp
    L.dgm_instance_replace.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(MeshDesc), ctypes.POINTER(Params)]
    L.dgm_instance_capacity.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(SlotCapacity)]
    L.dgm_create_mixed.argtypes = [ctypes.c_int32, ctypes.POINTER(MeshDesc), P_I32, ctypes.POINTER(TablesDesc),
                                   ctypes.POINTER(Params), ctypes.POINTER(SlotCapacity), P_I32]
    L.dgm_create_mixed.restype = vp
    L.dgm_instance_upload.argtypes = [vp, ctypes.c_int32, P_D]
    L.dgm_instance_download.argtypes = [vp, ctypes.c_int32, P_D]
    L.dgm_instance_download_residual.argtypes = [vp, ctypes.c_int32, P_D]
    L.dgm_instance_state.argtypes = [vp, ctypes.c_int32, P_D, P_I64, P_I32, P_I64]
    L.dgm_instance_set.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_int64, ctypes.c_double,
                                   ctypes.c_int64]
    L.dgm_advance_with_residual.argtypes = [vp, ctypes.c_int64]
    L.dgm_set_initial_solution.argtypes = [vp] + [ctypes.c_double] * 4
    L.dgm_set_launch_config.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.dgm_get_launch_config.argtypes = [vp, P_I32]
    L.dgm_autotune.argtypes = [vp, ctypes.c_int32, P_D]
    L.dgm_set_limiter_variant.argtypes = [vp, ctypes.c_int32]
    L.dgm_cell_fields.argtypes = [vp, ctypes.c_int32, P_D]
    L.dgm_set_edge_variant.argtypes = [vp, ctypes.c_int32]
    L.dgm_get_edge_variant.argtypes = [vp]
    L.dgm_get_limiter_variant.argtypes = [vp, P_I32, P_D]
    L.dgm_set_limiter_schedule.argtypes = [vp, ctypes.c_int32]
    L.dgm_get_limiter_schedule.argtypes = [vp, P_I32, P_D]
    L.dgm_instance_set_initial.argtypes = [vp, ctypes.c_int32] + [ctypes.c_double] * 4
    L.dgm_diagnostics.argtypes = [vp, ctypes.c_int32, P_D]
    L.dgm_enqueue_diagnostics.argtypes = [vp, ctypes.c_int32]
    L.dgm_set_viscous.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, P_D]
    L.dgm_set_limiter_grid.argtypes = [vp, ctypes.c_int32]
    L.dgm_get_limiter_grid.argtypes = [vp]
    L.dgm_get_viscous.argtypes = [vp]
    L.dgm_collected_diagnostics.argtypes = [vp, P_D]
    L.dgm_precision.argtypes = [vp]
    L.dgm_upload_solutions.argtypes = [vp, P_D]
    L.dgm_download_solutions.argtypes = [vp, P_D]
    L.dgm_advance.argtypes = [vp, ctypes.c_int64]
    L.dgm_synchronize.argtypes = [vp]
    L.dgm_query.argtypes = [vp]
    L.dgm_stream.argtypes = [vp]
    L.dgm_stream.restype = vp
    L.dgm_error_location.argtypes = [vp]
    L.dgm_error_location.restype = ctypes.c_int64
    L.dgm_limiter_stats.argtypes = [vp, P_I64, P_I32]
    L.dgm_device_bytes.argtypes = [vp]
    L.dgm_device_bytes.restype = ctypes.c_int64
    L.dgm_status_string.argtypes = [ctypes.c_int32]
    L.dgm_status_string.restype = ctypes.c_char_p
    L.dgm_version.argtypes = []
    L.dgm_version.restype = ctypes.c_char_p
    L.dgm_mesh_process.argtypes = [ctypes.c_int64, P_D, ctypes.c_int64, P_I64, ctypes.c_int64, P_I64, P_I32]
    L.dgm_mesh_process.restype = vp
    L.dgm_mesh_counts.argtypes = [vp, P_I64, P_I64, P_I64]
    L.dgm_mesh_counts.restype = ctypes.c_int32
    L.dgm_mesh_fetch.argtypes = [vp, P_I64, P_I64, P_D, P_D, P_D, P_I64, P_I64, P_I64, P_D, P_D, P_I64, P_I64, P_I64]
    L.dgm_mesh_fetch.restype = ctypes.c_int32
    L.dgm_mesh_free.argtypes = [vp]
    L.dgm_mesh_free.restype = None
    L.dgm_gmsh_parse.argtypes = [ctypes.c_char_p, P_I32]
    L.dgm_gmsh_parse.restype = vp
    L.dgm_gmsh_counts.argtypes = [vp, P_I64, P_I32, P_I32]
    L.dgm_gmsh_counts.restype = ctypes.c_int32
    L.dgm_gmsh_vertices.argtypes = [vp, P_D]
    L.dgm_gmsh_vertices.restype = ctypes.c_int32
    L.dgm_gmsh_block_size.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
    L.dgm_gmsh_block_size.restype = ctypes.c_int64
    L.dgm_gmsh_block_name.argtypes = [vp, ctypes.c_int32]
    L.dgm_gmsh_block_name.restype = ctypes.c_char_p
    L.dgm_gmsh_block.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, P_I64]
    L.dgm_gmsh_block.restype = ctypes.c_int32
    L.dgm_gmsh_free.argtypes = [vp]
    L.dgm_gmsh_free.restype = None
    L.dgm_vtk_write.argtypes = [ctypes.c_char_p, ctypes.c_int64, P_D, ctypes.c_int64, P_I64, P_D]
    L.dgm_vtk_write.restype = ctypes.c_int32
    for name in ("dgm_compute_residuals", "dgm_apply_limiter", "dgm_compute_time_step", "dgm_rk3",
                 "dgm_time_march", "dgm_get_clock", "dgm_set_clock", "dgm_upload_solutions",
                 "dgm_download_solutions", "dgm_advance", "dgm_synchronize", "dgm_query", "dgm_limiter_stats",
                 "dgm_set_limits", "dgm_launch_phase", "dgm_phase_launches_per_step", "dgm_launches_per_step",
                 "dgm_instance_count", "dgm_instance_upload", "dgm_instance_download",
                 "dgm_instance_download_residual", "dgm_instance_state", "dgm_instance_set",
                 "dgm_advance_with_residual", "dgm_diagnostics", "dgm_precision", "dgm_set_initial_solution",
                 "dgm_instance_set_initial", "dgm_set_launch_config", "dgm_get_launch_config", "dgm_autotune",
                 "dgm_set_limiter_variant", "dgm_get_limiter_variant", "dgm_set_limiter_schedule",
                 "dgm_get_limiter_schedule", "dgm_cell_fields", "dgm_set_edge_variant", "dgm_get_edge_variant",
                 "dgm_instance_replace", "dgm_instance_capacity", "dgm_enqueue_diagnostics",
                 "dgm_collected_diagnostics", "dgm_set_viscous", "dgm_get_viscous", "dgm_set_limiter_grid",
                 "dgm_get_limiter_grid"):
        getattr(L, name).restype = ctypes.c_int32
    _lib = L
    return L


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P_D)


def iptr(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(P_I64)


def i32ptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(P_I32)
