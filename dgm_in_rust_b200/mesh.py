"""Mesh ingest and preprocessing (host side, once per solve).

Restates the reference's mesh pipeline (the gmsh reader, the edge numbering and the geometry run
natively in the library; the O-grid generator and the gmsh writer are numpy):

* ``GmshParser.parse``   -- src/io/mesh_parser.rs:28-158 (gmsh 4.1 ASCII line state machine)
* ``process_mesh``       -- src/initialization.rs:112-261 (edge numbering, left/right rule,
  in-cell indices, internal/boundary lists)
* ``Mesh.compute_*``     -- src/mesh.rs:15-147 (edge length and normal, element Jacobian,
  circumradius, minimum height, neighbours)

plus a synthetic NACA 0012 O-grid generator that writes gmsh 4.1 files the reference parser
accepts (the reference ships no mesh for its configured ``naca0012.msh``).

Conventions that the device kernels rely on (all from the reference):
  * boundary edges are numbered first, block by block, then internal edges in order of first
    appearance over elements and their local edges (node pairs (v_i, v_{i+1 mod 3}));
  * an internal edge's left element is the one whose local vertex i equals the edge's first
    vertex; its normal (dy, -dx)/|e| points from left to right for counter-clockwise elements;
  * a boundary edge belongs to ``ielements[0]`` with ``ielements[1] == -1``.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import Sequence

import numpy as np

__all__ = [
    "BoundaryType",
    "EdgeBlock",
    "RawMesh",
    "Mesh",
    "GmshParser",
    "process_mesh",
    "naca0012_ogrid",
    "radial_distribution",
    "write_gmsh",
    "freestream_quantity",
]


class BoundaryType:
    WALL = 0
    FARFIELD = 1


@dataclasses.dataclass
class EdgeBlock:
    """One boundary line block: node pairs (0-based) and its physical name (mesh_parser.rs:5-8)."""

    node_pairs: np.ndarray
    physical_name: str


@dataclasses.dataclass
class RawMesh:
    """What GmshParser::parse returns: vertices, boundary edge blocks, triangle blocks."""

    vertices: np.ndarray                 # [nv, 2]
    edge_blocks: list                    # list[EdgeBlock]
    element_blocks: list                 # list[np.ndarray [n, 3]] 0-based node ids


class GmshParser:
    """gmsh 4.1 ASCII reader with the reference's state machine (mesh_parser.rs:28-158), run
    natively by the library (dgm_gmsh_parse).

    Quirks kept: every 3-token line inside $Nodes is a coordinate line (node tags are taken as
    file order); an entity is registered only from lines with at least 11 tokens (curves and
    surfaces); element blocks of dimension other than 1 or 2 are not expected.  Where the
    reference panics (a missing file, a malformed number, an entity without a physical name) this
    raises DgmError (DGM_BAD_ARG).
    """

    @staticmethod
    def parse(filename: str) -> RawMesh:
        from . import _native
        L = _native.lib()
        st = ctypes.c_int32(0)
        h = L.dgm_gmsh_parse(str(filename).encode(), ctypes.byref(st))
        if not h:
            raise _native.DgmError(st.value, what=f"GmshParser.parse({filename})")
        try:
            nv, neb, nel = ctypes.c_int64(0), ctypes.c_int32(0), ctypes.c_int32(0)
            L.dgm_gmsh_counts(h, ctypes.byref(nv), ctypes.byref(neb), ctypes.byref(nel))
            xy = np.empty((nv.value, 2))
            if nv.value:
                L.dgm_gmsh_vertices(h, _native.dptr(xy))
            edge_blocks, elem_blocks = [], []
            for i in range(neb.value):
                pairs = np.empty((L.dgm_gmsh_block_size(h, 1, i), 2), np.int64)
                if pairs.size:
                    L.dgm_gmsh_block(h, 1, i, _native.iptr(pairs))
                edge_blocks.append(EdgeBlock(pairs, L.dgm_gmsh_block_name(h, i).decode()))
            for i in range(nel.value):
                tris = np.empty((L.dgm_gmsh_block_size(h, 2, i), 3), np.int64)
                if tris.size:
                    L.dgm_gmsh_block(h, 2, i, _native.iptr(tris))
                elem_blocks.append(tris)
        finally:
            L.dgm_gmsh_free(h)
        return RawMesh(vertices=xy, edge_blocks=edge_blocks, element_blocks=elem_blocks)


def freestream_quantity(mach: float, aoa_deg: float, rho: float, p: float, hcr: float) -> np.ndarray:
    """BoundaryQuantity {rho, u, v, p} of a far-field patch (initialization.rs:125-132)."""
    c = math.sqrt(hcr * p / rho)
    a = aoa_deg * (math.pi / 180.0)
    return np.array([rho, mach * c * math.cos(a), mach * c * math.sin(a), p], dtype=np.float64)


@dataclasses.dataclass
class Mesh:
    """Mesh / Element / Edge / Patch of mesh.rs:5-189 as dense arrays."""

    vertices: np.ndarray            # [nv, 2]
    elem_vertices: np.ndarray       # [ne, 3] Element::ivertices
    elem_edges: np.ndarray          # [ne, 3] Element::iedges
    elem_neighbours: np.ndarray     # [ne, 3] Element::ineighbours (-1: none)
    elem_jacob_det: np.ndarray      # [ne]
    elem_circumradius: np.ndarray   # [ne]
    elem_minimum_height: np.ndarray # [ne]
    edge_elements: np.ndarray       # [ned, 2] Edge::ielements
    edge_vertices: np.ndarray       # [ned, 2] Edge::ivertices
    edge_in_cell: np.ndarray        # [ned, 2] Edge::in_cell_indices
    edge_jacob_det: np.ndarray      # [ned]
    edge_normal: np.ndarray         # [ned, 2]
    edge_patch: np.ndarray          # [ned] Edge::ipatch
    patch_type: np.ndarray          # [np] BoundaryType
    patch_quantity: np.ndarray      # [np, 4] rho, u, v, p (zeros for walls)
    internal_edge_indices: np.ndarray
    internal_element_indices: np.ndarray
    boundary_element_indices: np.ndarray

    @property
    def n_elements(self) -> int:
        return int(self.elem_vertices.shape[0])

    @property
    def n_edges(self) -> int:
        return int(self.edge_vertices.shape[0])

    def elem_inverse_jacobian(self) -> np.ndarray:
        """[ne, 4] (dxi/dx, dxi/dy, deta/dx, deta/dy) of compute_dphi (mesh.rs:93-100)."""
        v = self.vertices
        iv = self.elem_vertices
        x1, x2, x3 = v[iv[:, 0], 0], v[iv[:, 1], 0], v[iv[:, 2], 0]
        y1, y2, y3 = v[iv[:, 0], 1], v[iv[:, 1], 1], v[iv[:, 2], 1]
        J = self.elem_jacob_det
        return np.stack([(y3 - y1) / J, -(x3 - x1) / J, -(y2 - y1) / J, (x2 - x1) / J], axis=1)


def process_mesh(raw: RawMesh, freestream: np.ndarray, hcr: float) -> Mesh:
    """process_mesh (initialization.rs:112-261) followed by the Mesh::compute_* geometry of
    initialize_mesh_basis_gauss_params (initialization.rs:59-65).

    The edge numbering, element-edge assignment, geometry and neighbours are computed natively
    by the library (dgm_mesh_process: one pass, linear in the mesh size).  ``freestream`` is the
    far-field BoundaryQuantity (rho, u, v, p) given to every "Farfield" block; "Wall" blocks get
    none; any other name is rejected like the reference's panic.
    """
    from . import _native
    xy = np.ascontiguousarray(raw.vertices, dtype=np.float64)
    nv = xy.shape[0]
    ev_list, ep_list, ptype, pq = [], [], [], []
    for blk in raw.edge_blocks:
        name = blk.physical_name.lower()
        if name == "wall":
            ptype.append(BoundaryType.WALL)
            pq.append(np.zeros(4))
        elif name == "farfield":
            ptype.append(BoundaryType.FARFIELD)
            pq.append(np.asarray(freestream, dtype=np.float64))
        else:
            raise ValueError("Boundary type not implemented")
        ev_list.append(np.asarray(blk.node_pairs, dtype=np.int64).reshape(-1, 2))
        ep_list.append(np.full(len(blk.node_pairs), len(ptype) - 1, dtype=np.int64))
    bverts = np.ascontiguousarray(np.concatenate(ev_list) if ev_list else np.zeros((0, 2), np.int64))
    bpatch = np.concatenate(ep_list) if ep_list else np.zeros(0, np.int64)
    nbd = bverts.shape[0]
    blocks = [np.asarray(t, dtype=np.int64).reshape(-1, 3) for t in raw.element_blocks]
    elem_vertices = np.ascontiguousarray(np.concatenate(blocks) if blocks else np.zeros((0, 3), np.int64))
    ne = elem_vertices.shape[0]

    L = _native.lib()
    st = ctypes.c_int32(0)
    h = L.dgm_mesh_process(nv, _native.dptr(xy), nbd, _native.iptr(bverts), ne, _native.iptr(elem_vertices),
                           ctypes.byref(st))
    if not h:
        raise _native.DgmError(st.value, what="process_mesh")
    try:
        ned, nie, nil = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        L.dgm_mesh_counts(h, ctypes.byref(ned), ctypes.byref(nie), ctypes.byref(nil))
        ned, nie, nil = ned.value, nie.value, nil.value
        elem_edges, nbr = np.empty((ne, 3), np.int64), np.empty((ne, 3), np.int64)
        jac, circ, hmin = np.empty(ne), np.empty(ne), np.empty(ne)
        edge_elements, edge_vertices = np.empty((ned, 2), np.int64), np.empty((ned, 2), np.int64)
        edge_in_cell, edge_jac, edge_normal = np.empty((ned, 2), np.int64), np.empty(ned), np.empty((ned, 2))
        internal_edges, internal_el = np.empty(nie, np.int64), np.empty(nil, np.int64)
        boundary_el = np.empty(ne - nil, np.int64)
        P = _native.iptr
        D = _native.dptr
        L.dgm_mesh_fetch(h, P(elem_edges), P(nbr), D(jac), D(circ), D(hmin), P(edge_elements), P(edge_vertices),
                         P(edge_in_cell), D(edge_jac), D(edge_normal), P(internal_edges), P(internal_el),
                         P(boundary_el))
    finally:
        L.dgm_mesh_free(h)
    edge_patch = np.full(ned, -1, np.int64)
    edge_patch[:nbd] = bpatch
    return Mesh(
        vertices=xy,
        elem_vertices=elem_vertices,
        elem_edges=elem_edges,
        elem_neighbours=nbr,
        elem_jacob_det=jac,
        elem_circumradius=circ,
        elem_minimum_height=hmin,
        edge_elements=edge_elements,
        edge_vertices=edge_vertices,
        edge_in_cell=edge_in_cell,
        edge_jacob_det=edge_jac,
        edge_normal=edge_normal,
        edge_patch=edge_patch,
        patch_type=np.array(ptype, dtype=np.int32),
        patch_quantity=np.array(pq, dtype=np.float64).reshape(-1, 4),
        internal_edge_indices=internal_edges,
        internal_element_indices=internal_el,
        boundary_element_indices=boundary_el,
    )


# ---------------------------------------------------------------------------------------------
# Synthetic NACA 0012 O-grid
# ---------------------------------------------------------------------------------------------
def _naca0012_half_thickness(x: np.ndarray) -> np.ndarray:
    # closed trailing edge (last coefficient -0.1036)
    return 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def radial_distribution(nj: int, stretch: float = 1.15, radius: float = 20.0,
                        min_spacing: float = 1.0e-8) -> np.ndarray:
    """Normalised radial stations s_0 = 0 < ... < s_nj = 1, geometric with ratio ``stretch``.

    When that ratio would make the first spacing (s_1 * radius) smaller than ``min_spacing``
    chords -- from nj of about 130 up at ratio 1.15, e.g. 1e-31 chords at nj = 512, below the
    FP64 resolution of the vertex coordinates -- the ratio is lowered (bisection) until the first
    spacing equals ``min_spacing``."""
    def first(r):
        return (r - 1.0) / (r ** nj - 1.0) if r != 1.0 else 1.0 / nj
    r = stretch
    if stretch > 1.0 and first(stretch) * radius < min_spacing:
        lo, hi = 1.0 + 1e-12, stretch
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if first(mid) * radius < min_spacing:
                hi = mid
            else:
                lo = mid
        r = lo
    if r == 1.0:
        return np.arange(nj + 1) / nj
    return (r ** np.arange(nj + 1) - 1.0) / (r ** nj - 1.0)


def naca0012_ogrid(ni: int, nj: int, radius: float = 20.0, stretch: float = 1.15,
                   order: str = "colored", min_spacing: float = 1.0e-8) -> RawMesh:
    """NACA 0012 O-grid: ``ni`` quads around the airfoil, ``nj`` quads outward.

    Surface points use cosine clustering (x = (1 + cos th)/2, th = 2 pi i/ni, upper surface
    first, counter-clockwise); the far-field circle of ``radius`` chords is centred at mid
    chord; radial spacing grows geometrically by ``stretch`` with the first spacing chosen so
    the layers reach the circle.  Each quad (i, j) is split along the diagonal n(i,j)-n(i+1,j+1)
    into the counter-clockwise triangles A = (n00, n11, n10) and B = (n00, n01, n11).

    ``order="colored"`` numbers all A triangles, then all B triangles (each in radial-line
    order).  The dual graph is bipartite between A and B, so with this numbering every chain of
    increasing-index neighbours has length <= 2; ``order="quad"`` numbers A and B of each quad
    consecutively (the usual structured numbering).

    Returns the RawMesh that GmshParser would read from the written file (boundary blocks
    "Wall" (j = 0) then "Farfield" (j = nj), one triangle block).
    """
    if ni < 3 or nj < 1:
        raise ValueError("need ni >= 3, nj >= 1")
    th = 2.0 * np.pi * np.arange(ni) / ni
    xs = 0.5 * (1.0 + np.cos(th))
    ys = np.where(np.sin(th) >= 0.0, 1.0, -1.0) * _naca0012_half_thickness(np.clip(xs, 0.0, 1.0))
    xs[0], ys[0] = 1.0, 0.0
    ox = 0.5 + radius * np.cos(th)
    oy = radius * np.sin(th)
    sj = radial_distribution(nj, stretch, radius, min_spacing)
    X = (1.0 - sj)[:, None] * xs[None, :] + sj[:, None] * ox[None, :]
    Y = (1.0 - sj)[:, None] * ys[None, :] + sj[:, None] * oy[None, :]
    vertices = np.stack([X.reshape(-1), Y.reshape(-1)], axis=1)  # node (i, j) = j * ni + i

    def n(i, j):
        return j * ni + (i % ni)

    ii, jj = np.meshgrid(np.arange(ni), np.arange(nj), indexing="ij")  # radial lines contiguous
    ii, jj = ii.reshape(-1), jj.reshape(-1)
    n00, n10, n11, n01 = n(ii, jj), n(ii + 1, jj), n(ii + 1, jj + 1), n(ii, jj + 1)
    A = np.stack([n00, n11, n10], axis=1)
    B = np.stack([n00, n01, n11], axis=1)
    if order == "colored":
        tris = np.concatenate([A, B])
    elif order == "quad":
        tris = np.stack([A, B], axis=1).reshape(-1, 3)
    else:
        raise ValueError("order must be 'colored' or 'quad'")
    i = np.arange(ni)
    wall = np.stack([n(i, 0), n(i + 1, 0)], axis=1)
    far = np.stack([n(i, nj), n(i + 1, nj)], axis=1)
    raw = RawMesh(vertices=vertices, edge_blocks=[EdgeBlock(wall, "Wall"), EdgeBlock(far, "Farfield")],
                  element_blocks=[tris.astype(np.int64)])
    x, y = vertices[:, 0], vertices[:, 1]
    t = raw.element_blocks[0]
    jac = (x[t[:, 1]] - x[t[:, 0]]) * (y[t[:, 2]] - y[t[:, 0]]) - (x[t[:, 2]] - x[t[:, 0]]) * (y[t[:, 1]] - y[t[:, 0]])
    if not np.all(jac > 0.0):
        raise RuntimeError("O-grid produced a non counter-clockwise triangle")
    return raw


def write_gmsh(raw: RawMesh, path: str) -> None:
    """Write ``raw`` as gmsh 4.1 ASCII that GmshParser (and the reference's parser) reads back
    exactly: coordinates with 17 significant digits, distinct entity tags across dimensions,
    curve/surface entity lines of at least 11 tokens."""
    nv = raw.vertices.shape[0]
    names = [b.physical_name for b in raw.edge_blocks]
    lines = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(names) + 1)]
    for k, nm in enumerate(names):
        lines.append(f'1 {k + 1} "{nm}"')
    fluid_tag = len(names) + 1
    lines.append(f'2 {fluid_tag} "Fluid"')
    lines.append("$EndPhysicalNames")
    xmin, ymin = raw.vertices.min(axis=0)
    xmax, ymax = raw.vertices.max(axis=0)
    curve_tags = [100 + k for k in range(len(names))]
    surf_tag = 1000
    lines += ["$Entities", f"2 {len(names)} {len(raw.element_blocks)} 0",
              f"1 {xmin:.17g} {ymin:.17g} 0 0", f"2 {xmax:.17g} {ymax:.17g} 0 0"]
    for k, ct in enumerate(curve_tags):
        lines.append(f"{ct} {xmin:.17g} {ymin:.17g} 0 {xmax:.17g} {ymax:.17g} 0 1 {k + 1} 2 1 -2")
    for s in range(len(raw.element_blocks)):
        bound = " ".join(str(t) for t in curve_tags)
        lines.append(f"{surf_tag + s} {xmin:.17g} {ymin:.17g} 0 {xmax:.17g} {ymax:.17g} 0 1 {fluid_tag} "
                     f"{len(curve_tags)} {bound}")
    lines.append("$EndEntities")
    lines += ["$Nodes", f"1 {nv} 1 {nv}", f"2 {surf_tag} 0 {nv}"]
    lines += [str(i + 1) for i in range(nv)]
    lines += [f"{px:.17g} {py:.17g} 0" for px, py in raw.vertices]
    lines.append("$EndNodes")
    n_el = sum(len(b.node_pairs) for b in raw.edge_blocks) + sum(len(t) for t in raw.element_blocks)
    nblocks = len(raw.edge_blocks) + len(raw.element_blocks)
    lines += ["$Elements", f"{nblocks} {n_el} 1 {n_el}"]
    tag = 1
    for k, b in enumerate(raw.edge_blocks):
        lines.append(f"1 {curve_tags[k]} 1 {len(b.node_pairs)}")
        for p in b.node_pairs:
            lines.append(f"{tag} {p[0] + 1} {p[1] + 1}")
            tag += 1
    for s, t in enumerate(raw.element_blocks):
        lines.append(f"2 {surf_tag + s} 2 {len(t)}")
        for tri in t:
            lines.append(f"{tag} {tri[0] + 1} {tri[1] + 1} {tri[2] + 1}")
            tag += 1
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
