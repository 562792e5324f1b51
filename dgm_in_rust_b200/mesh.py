"""Mesh ingest and preprocessing (host side, once per solve).

Restates, vectorised with numpy, the reference's mesh pipeline:

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
    """gmsh 4.1 ASCII reader with the reference's state machine (mesh_parser.rs:28-158).

    Quirks kept: every 3-token line inside $Nodes is a coordinate line (node tags are taken as
    file order); an entity is registered only from lines with at least 11 tokens (curves and
    surfaces); element blocks of dimension other than 1 or 2 are not expected.
    """

    @staticmethod
    def parse(filename: str) -> RawMesh:
        physical_names: dict[int, str] = {}
        ent_to_phys: dict[int, int] = {}
        xy: list[float] = []
        edge_blocks: list[tuple[list[int], str]] = []
        elem_blocks: list[list[int]] = []
        state = "standby"
        line_count = max_line_count = 0
        with open(filename, "r") as f:
            for raw in f:
                line = raw.rstrip("\r\n")
                if line.startswith("$End"):
                    state = "standby"
                    continue
                if line.startswith("$PhysicalNames"):
                    state = "first_phys"
                    continue
                if line.startswith("$Entities"):
                    state = "first_ent"
                    continue
                if line.startswith("$Nodes"):
                    state = "first_nodes"
                    continue
                if line.startswith("$Elements"):
                    state = "first_elems"
                    continue
                v = line.split()
                if state == "standby":
                    continue
                if state == "first_phys":
                    state = "phys"
                elif state == "phys":
                    if len(v) == 3:
                        physical_names[int(v[1])] = v[2].strip('"')
                elif state == "first_ent":
                    state = "ent"
                elif state == "ent":
                    if len(v) >= 11:
                        ent_to_phys[int(v[0])] = int(v[8])
                elif state == "first_nodes":
                    state = "nodes"
                elif state == "nodes":
                    if len(v) == 3:
                        xy.append(float(v[0]))
                        xy.append(float(v[1]))
                elif state == "first_elems":
                    state = "first_block"
                elif state == "first_block":
                    dim, tag, num = int(v[0]), int(v[1]), int(v[3])
                    name = physical_names[ent_to_phys[tag]]
                    if dim == 1:
                        edge_blocks.append(([], name))
                        state = "edge_block"
                    if dim == 2:
                        elem_blocks.append([])
                        state = "elem_block"
                    line_count, max_line_count = 0, num
                elif state == "edge_block":
                    line_count += 1
                    edge_blocks[-1][0].extend((int(v[1]) - 1, int(v[2]) - 1))
                    if line_count == max_line_count:
                        state = "first_block"
                elif state == "elem_block":
                    line_count += 1
                    elem_blocks[-1].extend((int(v[1]) - 1, int(v[2]) - 1, int(v[3]) - 1))
                    if line_count == max_line_count:
                        state = "first_block"
        return RawMesh(
            vertices=np.array(xy, dtype=np.float64).reshape(-1, 2),
            edge_blocks=[EdgeBlock(np.array(p, dtype=np.int64).reshape(-1, 2), n) for p, n in edge_blocks],
            element_blocks=[np.array(b, dtype=np.int64).reshape(-1, 3) for b in elem_blocks],
        )


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


def _assign_sequential(e_base, tris, edge_ids, edge_vertices, edge_elements, edge_in_cell):
    """The reference's element->edge assignment loop (initialization.rs:181-201), used only when
    a mesh has repeated (edge, side) writes and the vectorised path would be ambiguous."""
    internal = np.ones(tris.shape[0], dtype=bool)
    for t in range(tris.shape[0]):
        e = e_base + t
        for k in range(3):
            d = edge_ids[t, k]
            if edge_elements[d, 1] == -1:
                edge_elements[d, 0] = e
                edge_in_cell[d, 0] = k
                internal[t] = False
            elif tris[t, k] == edge_vertices[d, 0]:
                edge_elements[d, 0] = e
                edge_in_cell[d, 0] = k
            else:
                edge_elements[d, 1] = e
                edge_in_cell[d, 1] = k
    return internal


def process_mesh(raw: RawMesh, freestream: np.ndarray, hcr: float) -> Mesh:
    """process_mesh (initialization.rs:112-261) followed by the Mesh::compute_* geometry of
    initialize_mesh_basis_gauss_params (initialization.rs:59-65).

    ``freestream`` is the far-field BoundaryQuantity (rho, u, v, p) given to every "Farfield"
    block; "Wall" blocks get none; any other name is rejected like the reference's panic.
    """
    xy = np.ascontiguousarray(raw.vertices, dtype=np.float64)
    nv = xy.shape[0]
    key_of = lambda pairs: np.minimum(pairs[:, 0], pairs[:, 1]) * nv + np.maximum(pairs[:, 0], pairs[:, 1])
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
    bverts = np.concatenate(ev_list) if ev_list else np.zeros((0, 2), np.int64)
    bpatch = np.concatenate(ep_list) if ep_list else np.zeros(0, np.int64)
    nbd = bverts.shape[0]
    # edge map: unordered node pair -> edge id (lookups try (a,b) then (b,a))
    emap_keys = key_of(bverts) if nbd else np.zeros(0, np.int64)
    emap_ids = np.arange(nbd, dtype=np.int64)
    if nbd:  # a repeated pair maps to its last insertion
        order = np.argsort(emap_keys, kind="stable")
        k_sorted = emap_keys[order]
        last = np.r_[k_sorted[1:] != k_sorted[:-1], True]
        emap_keys, emap_ids = k_sorted[last], emap_ids[order][last]
    edge_vertices = [bverts]
    n_edges = nbd
    internal_edges = []
    elem_vertices, elem_edges, internal_flags = [], [], []
    # grow-only arrays for ielements / in_cell_indices
    cap = nbd + 3 * sum(b.shape[0] for b in raw.element_blocks)
    edge_elements = np.zeros((cap, 2), np.int64)
    edge_in_cell = np.zeros((cap, 2), np.int64)
    edge_elements[:nbd] = (0, -1)
    edge_in_cell[:nbd] = (0, -1)
    e_base = 0
    for tris in raw.element_blocks:
        tris = np.asarray(tris, dtype=np.int64).reshape(-1, 3)
        nt = tris.shape[0]
        pairs = np.stack([tris, np.roll(tris, -1, axis=1)], axis=2).reshape(-1, 2)  # (v_i, v_{i+1})
        keys = key_of(pairs)
        pos = np.searchsorted(emap_keys, keys)
        pos_c = np.minimum(pos, max(len(emap_keys) - 1, 0))
        found = (len(emap_keys) > 0) & (emap_keys[pos_c] == keys) if len(emap_keys) else np.zeros(len(keys), bool)
        # new internal edges, numbered by first appearance
        new_keys, first_idx = np.unique(keys[~found], return_index=True)
        cand = np.nonzero(~found)[0]
        first_pos = cand[first_idx]
        order = np.argsort(first_pos, kind="stable")
        new_keys, first_pos = new_keys[order], first_pos[order]
        new_ids = n_edges + np.arange(len(new_keys), dtype=np.int64)
        edge_vertices.append(pairs[first_pos])
        internal_edges.append(new_ids)
        edge_elements[n_edges:n_edges + len(new_keys)] = 0
        edge_in_cell[n_edges:n_edges + len(new_keys)] = 0
        n_edges += len(new_keys)
        all_keys = np.concatenate([emap_keys, new_keys])
        all_ids = np.concatenate([emap_ids, new_ids])
        srt = np.argsort(all_keys, kind="stable")
        emap_keys, emap_ids = all_keys[srt], all_ids[srt]
        ids = emap_ids[np.searchsorted(emap_keys, keys)].reshape(nt, 3)
        ev_all = np.concatenate(edge_vertices)
        # assignment (initialization.rs:181-201)
        elem_idx = e_base + np.repeat(np.arange(nt, dtype=np.int64), 3)
        kk = np.tile(np.arange(3, dtype=np.int64), nt)
        flat = ids.reshape(-1)
        is_bnd = flat < nbd
        same = pairs[:, 0] == ev_all[flat, 0]
        left = is_bnd | same
        tgt_side = np.where(left, 0, 1)
        slot = flat * 2 + tgt_side
        if len(np.unique(slot)) != len(slot):
            internal = _assign_sequential(e_base, tris, ids, ev_all, edge_elements, edge_in_cell)
        else:
            edge_elements[flat, tgt_side] = elem_idx
            edge_in_cell[flat, tgt_side] = kk
            internal = ~is_bnd.reshape(nt, 3).any(axis=1)
        elem_vertices.append(tris)
        elem_edges.append(ids)
        internal_flags.append(internal)
        e_base += nt
    edge_vertices = np.concatenate(edge_vertices)
    edge_elements = edge_elements[:n_edges].copy()
    edge_in_cell = edge_in_cell[:n_edges].copy()
    edge_patch = np.full(n_edges, -1, np.int64)
    edge_patch[:nbd] = bpatch
    elem_vertices = np.concatenate(elem_vertices) if elem_vertices else np.zeros((0, 3), np.int64)
    elem_edges = np.concatenate(elem_edges) if elem_edges else np.zeros((0, 3), np.int64)
    internal_flags = np.concatenate(internal_flags) if internal_flags else np.zeros(0, bool)
    ne = elem_vertices.shape[0]

    # ---- geometry, mesh.rs:15-84 (same operation order as the reference) ----
    x, y = xy[:, 0], xy[:, 1]
    ex1, ex2 = x[edge_vertices[:, 0]], x[edge_vertices[:, 1]]
    ey1, ey2 = y[edge_vertices[:, 0]], y[edge_vertices[:, 1]]
    edx, edy = ex2 - ex1, ey2 - ey1
    edge_jac = np.sqrt(edx * edx + edy * edy)
    edge_normal = np.stack([edy / edge_jac, -edx / edge_jac], axis=1)
    x1, x2, x3 = x[elem_vertices[:, 0]], x[elem_vertices[:, 1]], x[elem_vertices[:, 2]]
    y1, y2, y3 = y[elem_vertices[:, 0]], y[elem_vertices[:, 1]], y[elem_vertices[:, 2]]
    jac = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)
    a = np.sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1))
    b = np.sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2))
    c = np.sqrt((x1 - x3) * (x1 - x3) + (y1 - y3) * (y1 - y3))
    s = (a + b + c) / 2.0
    with np.errstate(invalid="ignore", divide="ignore"):
        circ = a * b * c / (4.0 * np.sqrt(s * (s - a) * (s - b) * (s - c)))
        surface = 0.5 * jac
        hmin = np.fmin(np.fmin(2.0 * surface / a, 2.0 * surface / b), 2.0 * surface / c)
    # set_neighbours, mesh.rs:133-147
    nbr = np.full((ne, 3), -1, np.int64)
    d = elem_edges
    bnd = edge_elements[d, 1] == -1
    same = elem_vertices == edge_vertices[d, 0]
    other = np.where(same, edge_elements[d, 1], edge_elements[d, 0])
    nbr[~bnd] = other[~bnd]
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
        internal_edge_indices=np.concatenate(internal_edges) if internal_edges else np.zeros(0, np.int64),
        internal_element_indices=np.nonzero(internal_flags)[0].astype(np.int64),
        boundary_element_indices=np.nonzero(~internal_flags)[0].astype(np.int64),
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
