"""Result output in the reference's format: write_to_vtk (src/io/write_results.rs:8-93).

The reference writes, after the time loop (temporal_disc.rs:56), one legacy ASCII VTK file
``outputfiles/solutions/step=<current_step>.vtk`` through the vtkio crate: the vertices as points
(z = 0), the triangles, and three cell attributes computed from each element's mode-0
coefficients -- Density, Velocity (u, v, 0) and Pressure.  The cell fields come from the device
(``dgm_cell_fields``, bit-identical to the reference's expressions); the library writes the text
(``dgm_vtk_write``) exactly as vtkio's legacy writer does (empty title, each data block on one line, one cell
type per line, an empty POINT_DATA block) with numbers in Rust's ``{}`` form for f64 (shortest
round-trip digits, positional notation, no trailing ".0", ``NaN``/``inf``).
"""
from __future__ import annotations

import os

import numpy as np

__all__ = ["format_f64", "vtk_text", "write_to_vtk", "solution_path"]

_TRIANGLE = 5  # VTK cell type of a triangle


def format_f64(x: float) -> str:
    """Rust's Display of an f64."""
    x = float(x)
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    return np.format_float_positional(x, unique=True, trim="-")


def _join(values) -> str:
    return " ".join(format_f64(v) for v in values)


def vtk_text(vertices: np.ndarray, triangles: np.ndarray, fields: np.ndarray) -> str:
    """The file content: vertices [nv, 2], triangles [ne, 3] (vertex indices), fields [ne, 4] =
    density, x velocity, y velocity, pressure."""
    nv, ne = int(vertices.shape[0]), int(triangles.shape[0])
    if fields.shape != (ne, 4):
        raise ValueError("fields must be [n_elements, 4]")
    pts = np.zeros((nv, 3))
    pts[:, :2] = vertices
    cells = " ".join(f"3 {a} {b} {c}" for a, b, c in np.asarray(triangles, dtype=np.int64))
    vel = np.zeros((ne, 3))
    vel[:, :2] = fields[:, 1:3]
    lines = ["# vtk DataFile Version 2.0", "", "ASCII", "", "DATASET UNSTRUCTURED_GRID",
             f"POINTS {nv} double", _join(pts.reshape(-1)), "",
             f"CELLS {ne} {4 * ne}", cells, "",
             f"CELL_TYPES {ne}"] + [str(_TRIANGLE)] * ne + ["", "",
             f"POINT_DATA {nv}", "", f"CELL_DATA {ne}", "",
             "SCALARS Density double 1", "LOOKUP_TABLE default", _join(fields[:, 0]), "",
             "VECTORS Velocity double", _join(vel.reshape(-1)), "",
             "SCALARS Pressure double 1", "LOOKUP_TABLE default", _join(fields[:, 3]), ""]
    return "\n".join(lines) + "\n"


def solution_path(current_step: int, root: str = "outputfiles/solutions") -> str:
    """The reference's output file name (write_results.rs:85-91)."""
    return os.path.join(root, f"step={int(current_step)}.vtk")


def write_to_vtk(path: str, mesh, fields: np.ndarray) -> str:
    """Write the VTK file of ``mesh`` (a processed Mesh: vertices, elem_vertices) with the cell
    fields [ne, 4]; creates the directory like the reference.  The text is produced natively by
    the library (dgm_vtk_write), byte for byte what :func:`vtk_text` lays out.  Returns the path."""
    from . import _native
    xy = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    tris = np.ascontiguousarray(mesh.elem_vertices, dtype=np.int64)
    f = np.ascontiguousarray(fields, dtype=np.float64)
    if f.shape != (tris.shape[0], 4):
        raise ValueError("fields must be [n_elements, 4]")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    st = _native.lib().dgm_vtk_write(str(path).encode(), xy.shape[0], _native.dptr(xy), tris.shape[0],
                                     _native.iptr(tris), _native.dptr(f))
    if st != 0:
        raise _native.DgmError(st, what=f"write_to_vtk({path})")
    return path
