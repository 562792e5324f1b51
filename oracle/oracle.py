"""ctypes wrapper of the CPU oracle (oracle/dgm_oracle.cpp -> oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
arm as the checker.  The product package never imports this module.

Parity status: unpinned by reference outputs (the Rust reference cannot be built here and ships
no tests or golden vectors); see the header of dgm_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "liboracle.so")

P_D = ctypes.POINTER(ctypes.c_double)
P_I64 = ctypes.POINTER(ctypes.c_int64)
P_I32 = ctypes.POINTER(ctypes.c_int32)


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int32), ("ncell_gp", ctypes.c_int32), ("nedge_gp", ctypes.c_int32),
        ("limiter", ctypes.c_int32), ("threads", ctypes.c_int32), ("_pad", ctypes.c_int32),
        ("hcr", ctypes.c_double), ("cfl", ctypes.c_double), ("final_time", ctypes.c_double),
        ("final_step", ctypes.c_int64),
        ("fs_aoa_deg", ctypes.c_double), ("fs_mach", ctypes.c_double), ("fs_rho", ctypes.c_double),
        ("fs_p", ctypes.c_double),
        ("in_aoa_deg", ctypes.c_double), ("in_mach", ctypes.c_double), ("in_rho", ctypes.c_double),
        ("in_p", ctypes.c_double),
    ]


class OrcRawMesh(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int64), ("xy", P_D),
        ("n_edge_blocks", ctypes.c_int32), ("edge_block_sizes", P_I64), ("edge_block_types", P_I32),
        ("edge_pairs", P_I64),
        ("n_tri_blocks", ctypes.c_int32), ("tri_block_sizes", P_I64), ("tris", P_I64),
    ]


STATUS = {0: "ok", 1: "Negative density found in HLLC!", 2: "Negative pressure found in HLLC!",
          4: "Invalid number of boundary neighbours!", 7: "bad argument", 8: "parse error"}


class OracleError(RuntimeError):
    def __init__(self, status, where=-1):
        self.status = status
        self.where = where
        super().__init__(f"oracle: {STATUS.get(status, status)} (at {where})")


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.orc_create_from_msh.argtypes = [ctypes.c_char_p, ctypes.POINTER(OrcConfig), P_I32]
        L.orc_create_from_msh.restype = vp
        L.orc_create_from_raw.argtypes = [ctypes.POINTER(OrcRawMesh), ctypes.POINTER(OrcConfig), P_I32]
        L.orc_create_from_raw.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_sizes.argtypes = [vp, P_I64]
        L.orc_cfl.argtypes = [vp]
        L.orc_cfl.restype = ctypes.c_double
        L.orc_get_array.argtypes = [vp, ctypes.c_char_p, ctypes.c_void_p]
        L.orc_get_array.restype = ctypes.c_int32
        L.orc_element_dphi.argtypes = [vp, ctypes.c_int64, P_D]
        L.orc_set_initial_solution.argtypes = [vp, P_D]
        L.orc_compute_residuals.argtypes = [vp, P_D, P_D]
        L.orc_compute_residuals.restype = ctypes.c_int32
        L.orc_apply_limiter.argtypes = [vp, P_D, P_I64]
        L.orc_apply_limiter.restype = ctypes.c_int32
        L.orc_troubled_flags.argtypes = [vp, P_D, ctypes.POINTER(ctypes.c_int8)]
        L.orc_compute_time_step.argtypes = [vp, P_D]
        L.orc_compute_time_step.restype = ctypes.c_double
        L.orc_rk3.argtypes = [vp, P_D, P_D, ctypes.c_double]
        L.orc_rk3.restype = ctypes.c_int32
        L.orc_err_where.argtypes = [vp]
        L.orc_err_where.restype = ctypes.c_int64
        L.orc_time_march.argtypes = [vp, P_D, P_D, P_D, P_I64]
        L.orc_time_march.restype = ctypes.c_int32
        L.orc_reset_clock.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, ctypes.c_int32]
        L.orc_set_viscous.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double]
        L.orc_hllc.argtypes = [P_D, P_D, ctypes.c_double, ctypes.c_double, ctypes.c_double, P_D]
        L.orc_hllc.restype = ctypes.c_int32
        L.orc_flux.argtypes = [P_D, ctypes.c_double, P_D, P_D]
        L.orc_eigenmatrix.argtypes = [P_D, ctypes.c_double, ctypes.c_double, ctypes.c_double, P_D, P_D]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(P_D)


def hllc(lv, rv, nx, ny, hcr=1.4):
    """flux::hllc of one interface state pair; returns (status, flux[4])."""
    lv, rv, out = np.ascontiguousarray(lv, np.float64), np.ascontiguousarray(rv, np.float64), np.zeros(4)
    st = lib().orc_hllc(_d(lv), _d(rv), float(nx), float(ny), float(hcr), _d(out))
    return int(st), out


def euler_flux(q, hcr=1.4):
    q, f, g = np.ascontiguousarray(q, np.float64), np.zeros(4), np.zeros(4)
    lib().orc_flux(_d(q), float(hcr), _d(f), _d(g))
    return f, g


def eigenmatrix(q, nx, ny, hcr=1.4):
    q, L, R = np.ascontiguousarray(q, np.float64), np.zeros((4, 4)), np.zeros((4, 4))
    lib().orc_eigenmatrix(_d(q), float(nx), float(ny), float(hcr), _d(L), _d(R))
    return L, R


class Oracle:
    """One CPU restatement of the reference solver for one mesh."""

    def __init__(self, raw=None, msh_path=None, order=2, ncell_gp=6, nedge_gp=3, hcr=1.4, cfl=0.1,
                 final_time=1.0e30, final_step=1, limiter=True, threads=1, freestream=(1.25, 0.8, 1.0, 1.0 / 1.4),
                 initial=None):
        """``freestream``/``initial`` are (aoa_deg, mach, rho, p); ``raw`` is a RawMesh-like object with
        ``vertices``, ``edge_blocks`` (``node_pairs``, ``physical_name``) and ``element_blocks``."""
        L = lib()
        initial = initial if initial is not None else freestream
        cfg = OrcConfig(order=order, ncell_gp=ncell_gp, nedge_gp=nedge_gp, limiter=1 if limiter else 0,
                        threads=threads, _pad=0, hcr=hcr, cfl=cfl, final_time=final_time, final_step=final_step,
                        fs_aoa_deg=freestream[0], fs_mach=freestream[1], fs_rho=freestream[2], fs_p=freestream[3],
                        in_aoa_deg=initial[0], in_mach=initial[1], in_rho=initial[2], in_p=initial[3])
        st = ctypes.c_int32(0)
        if msh_path is not None:
            h = L.orc_create_from_msh(msh_path.encode(), ctypes.byref(cfg), ctypes.byref(st))
        else:
            xy = np.ascontiguousarray(raw.vertices, dtype=np.float64)
            eb_sizes = np.array([len(b.node_pairs) for b in raw.edge_blocks], dtype=np.int64)
            eb_types = np.array([0 if b.physical_name.lower() == "wall" else 1 for b in raw.edge_blocks], np.int32)
            pairs = np.ascontiguousarray(np.concatenate([np.asarray(b.node_pairs, np.int64).reshape(-1, 2)
                                                         for b in raw.edge_blocks]), dtype=np.int64)
            tb_sizes = np.array([len(t) for t in raw.element_blocks], dtype=np.int64)
            tris = np.ascontiguousarray(np.concatenate([np.asarray(t, np.int64).reshape(-1, 3)
                                                        for t in raw.element_blocks]), dtype=np.int64)
            self._keep = (xy, eb_sizes, eb_types, pairs, tb_sizes, tris)
            rm = OrcRawMesh(n_vertices=xy.shape[0], xy=_d(xy), n_edge_blocks=len(eb_sizes),
                            edge_block_sizes=eb_sizes.ctypes.data_as(P_I64),
                            edge_block_types=eb_types.ctypes.data_as(P_I32), edge_pairs=pairs.ctypes.data_as(P_I64),
                            n_tri_blocks=len(tb_sizes), tri_block_sizes=tb_sizes.ctypes.data_as(P_I64),
                            tris=tris.ctypes.data_as(P_I64))
            h = L.orc_create_from_raw(ctypes.byref(rm), ctypes.byref(cfg), ctypes.byref(st))
        if not h:
            raise OracleError(st.value)
        self._h = ctypes.c_void_p(h)
        self._L = L
        sz = np.zeros(12, np.int64)
        L.orc_sizes(self._h, sz.ctypes.data_as(P_I64))
        (self.ne, self.ned, self.nv, self.np_, self.nb, self.nq, self.ng, self.n_int_edges, self.n_int_elems,
         self.n_bnd_elems, self.nkeys, self.max_order) = [int(v) for v in sz]

    def close(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cfl(self) -> float:
        return float(self._L.orc_cfl(self._h))

    _SHAPES = {
        "xy": ("nv", 2, np.float64), "elem_vertices": ("ne", 3, np.int64), "elem_edges": ("ne", 3, np.int64),
        "elem_neighbours": ("ne", 3, np.int64), "elem_jacob_det": ("ne", 0, np.float64),
        "elem_circumradius": ("ne", 0, np.float64), "elem_minimum_height": ("ne", 0, np.float64),
        "elem_dinv": ("ne", 4, np.float64), "edge_elements": ("ned", 2, np.int64),
        "edge_vertices": ("ned", 2, np.int64), "edge_in_cell": ("ned", 2, np.int64),
        "edge_jacob_det": ("ned", 0, np.float64), "edge_normal": ("ned", 2, np.float64),
        "edge_patch": ("ned", 0, np.int64), "patch_quantity": ("np_", 4, np.float64),
        "patch_type": ("np_", 0, np.int64), "internal_edges": ("n_int_edges", 0, np.int64),
        "internal_elements": ("n_int_elems", 0, np.int64), "boundary_elements": ("n_bnd_elems", 0, np.int64),
    }

    def get(self, name: str) -> np.ndarray:
        if name in self._SHAPES:
            n, k, dt = self._SHAPES[name]
            shape = (getattr(self, n),) + ((k,) if k else ())
        elif name == "cell_points":
            shape, dt = (self.nq, 2), np.float64
        elif name == "cell_weights":
            shape, dt = (self.nq,), np.float64
        elif name == "edge_points":
            shape, dt = (3, self.ng, 2), np.float64
        elif name == "edge_weights":
            shape, dt = (self.ng,), np.float64
        elif name == "phi_cell":
            shape, dt = (self.nq, self.nb), np.float64
        elif name == "phi_edge":
            shape, dt = (3, self.ng, self.nb), np.float64
        elif name == "dphi_cell":
            shape, dt = (self.nq, self.nb, self.nkeys), np.float64
        elif name == "mass":
            shape, dt = (self.nb,), np.float64
        else:
            raise KeyError(name)
        out = np.zeros(shape, dtype=dt)
        if self._L.orc_get_array(self._h, name.encode(), out.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise KeyError(name)
        return out

    def element_dphi(self, e: int) -> np.ndarray:
        out = np.zeros((self.nq, self.nb, self.nkeys))
        self._L.orc_element_dphi(self._h, int(e), _d(out))
        return out

    def new_state(self):
        return np.zeros((self.ne, 4, self.nb))

    def initial_solution(self) -> np.ndarray:
        U = self.new_state()
        self._L.orc_set_initial_solution(self._h, _d(U))
        return U

    def _chk(self, st):
        if st != 0:
            raise OracleError(st, int(self._L.orc_err_where(self._h)))

    def compute_residuals(self, R: np.ndarray, U: np.ndarray) -> None:
        self._chk(self._L.orc_compute_residuals(self._h, _d(R), _d(U)))

    def apply_limiter(self, U: np.ndarray) -> int:
        n = ctypes.c_int64(0)
        self._chk(self._L.orc_apply_limiter(self._h, _d(U), ctypes.byref(n)))
        return int(n.value)

    def troubled_flags(self, U: np.ndarray) -> np.ndarray:
        f = np.zeros(self.ne, np.int8)
        self._L.orc_troubled_flags(self._h, _d(U), f.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)))
        return f

    def compute_time_step(self, U: np.ndarray) -> float:
        return float(self._L.orc_compute_time_step(self._h, _d(U)))

    def rk3(self, R: np.ndarray, U: np.ndarray, dt: float) -> None:
        self._chk(self._L.orc_rk3(self._h, _d(R), _d(U), float(dt)))

    def time_march(self, R: np.ndarray, U: np.ndarray):
        t, s = ctypes.c_double(0.0), ctypes.c_int64(0)
        self._chk(self._L.orc_time_march(self._h, _d(R), _d(U), ctypes.byref(t), ctypes.byref(s)))
        return float(t.value), int(s.value)

    def reset_clock(self):
        self._L.orc_reset_clock(self._h)

    def set_threads(self, n: int):
        self._L.orc_set_threads(self._h, int(n))

    def set_viscous(self, enable: bool = True, prandtl_number: float = 0.72, gas_constant: float = 287.0):
        """Navier-Stokes (BR2) residual in place of the Euler one: the reference's disabled
        integrate_over_cell_ns / integrate_over_edges_ns / apply_bc_ns (spatial_disc.rs:34-36)."""
        self._L.orc_set_viscous(self._h, 1 if enable else 0, float(prandtl_number), float(gas_constant))
