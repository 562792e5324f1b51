"""Host side of the product against the oracle, the gmsh round trip, and the C ABI library
(loads and exports every declared symbol; fails loudly without a GPU).  No GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, airfoil_raw
from dgm_in_rust_b200 import (DgmError, DubinerBasis, GaussPoints, GmshParser, InitialSolution, build_solver,
                              default_rules, freestream_quantity, initial_state, naca0012_ogrid, process_mesh,
                              write_gmsh)
from oracle.oracle import Oracle

FS = (1.25, 0.8, 1.0, 1.0 / 1.4)
MESH_FIELDS = [("elem_vertices", "elem_vertices"), ("elem_edges", "elem_edges"),
               ("elem_neighbours", "elem_neighbours"), ("elem_jacob_det", "elem_jacob_det"),
               ("elem_circumradius", "elem_circumradius"), ("elem_minimum_height", "elem_minimum_height"),
               ("edge_elements", "edge_elements"), ("edge_vertices", "edge_vertices"),
               ("edge_in_cell", "edge_in_cell"), ("edge_jacob_det", "edge_jacob_det"),
               ("edge_normal", "edge_normal"), ("edge_patch", "edge_patch"), ("patch_quantity", "patch_quantity"),
               ("internal_edges", "internal_edge_indices"), ("internal_elements", "internal_element_indices"),
               ("boundary_elements", "boundary_element_indices")]


def _fs_q(fs, hcr=1.4):
    return freestream_quantity(fs[1], fs[0], fs[2], fs[3], hcr)


def _check_mesh_equal(o, m):
    for oname, mname in MESH_FIELDS:
        a, b = o.get(oname), getattr(m, mname)
        assert a.shape == b.shape and np.array_equal(a, b), oname
    assert np.array_equal(o.get("elem_dinv"), m.elem_inverse_jacobian())


@pytest.mark.parametrize("ordering", ["colored", "quad"])
def test_process_mesh_matches_oracle_ogrid(ordering):
    raw = naca0012_ogrid(24, 12, order=ordering)
    m = process_mesh(raw, _fs_q(FS), 1.4)
    _check_mesh_equal(Oracle(raw=raw, order=2, freestream=FS), m)


def test_process_mesh_matches_oracle_airfoil():
    raw = airfoil_raw()
    fs = (1.5, 0.8, 1.0, 100000.0)
    m = process_mesh(raw, _fs_q(fs), 1.4)
    _check_mesh_equal(Oracle(raw=raw, order=2, freestream=fs), m)
    assert (m.elem_jacob_det > 0).all()  # every airfoil.msh triangle is counter-clockwise


def test_process_mesh_multiblock_repeated_pairs_matches_oracle():
    """Two triangle blocks and a boundary pair listed twice (reversed, in a second wall block):
    the edge numbering runs over the blocks in order and the repeated pair maps to its last
    listing, as the reference's HashMap insert does."""
    from dgm_in_rust_b200.mesh import EdgeBlock, RawMesh
    r = naca0012_ogrid(16, 8)
    t = r.element_blocks[0]
    wall, far = r.edge_blocks
    raw = RawMesh(r.vertices, [EdgeBlock(wall.node_pairs, "Wall"), EdgeBlock(wall.node_pairs[:3][:, ::-1].copy(), "Wall"),
                               EdgeBlock(far.node_pairs, "Farfield")], [t[:100].copy(), t[100:].copy()])
    m = process_mesh(raw, _fs_q(FS), 1.4)
    _check_mesh_equal(Oracle(raw=raw, order=2, freestream=FS), m)
    assert m.edge_elements[0, 0] == 0 and m.edge_elements[0, 1] == -1  # first listing never found


def test_process_mesh_larger_ogrid_matches_oracle():
    raw = naca0012_ogrid(128, 64, order="quad")
    m = process_mesh(raw, _fs_q(FS), 1.4)
    _check_mesh_equal(Oracle(raw=raw, order=2, freestream=FS), m)


def test_process_mesh_rejects_bad_node_index():
    from dgm_in_rust_b200.mesh import RawMesh
    r = naca0012_ogrid(8, 4)
    t = r.element_blocks[0].copy()
    t[5, 1] = r.vertices.shape[0]
    with pytest.raises(DgmError) as err:
        process_mesh(RawMesh(r.vertices, r.edge_blocks, [t]), _fs_q(FS), 1.4)
    assert err.value.status == 7  # DGM_BAD_ARG


@pytest.mark.parametrize("order", [1, 2, 3])
def test_tables_match_oracle(order):
    nq, ng = default_rules(order)
    g = GaussPoints(nq, ng)
    b = DubinerBasis(order, g)
    o = Oracle(raw=naca0012_ogrid(8, 4), order=order, ncell_gp=nq, nedge_gp=ng, freestream=FS)
    for name, mine in [("cell_points", g.cell_points), ("cell_weights", g.cell_weights),
                       ("edge_points", g.edge_points), ("edge_weights", g.edge_weights),
                       ("phi_cell", b.phis_cell_gps), ("phi_edge", b.phis_edge_gps), ("mass", b.mass_mat_diag)]:
        assert np.array_equal(o.get(name), mine), name
    d = o.get("dphi_cell")
    if order == 2:
        assert np.array_equal(d, b.dphis_cell_gps)  # the reference's closed forms, bit for bit
    else:
        assert np.allclose(d, b.dphis_cell_gps, rtol=1e-13, atol=1e-12)


def test_initial_state_matches_oracle():
    raw = naca0012_ogrid(16, 8)
    m = process_mesh(raw, _fs_q(FS), 1.4)
    g = GaussPoints(6, 3)
    b = DubinerBasis(2, g)
    U = initial_state(m, b, g, 1.4, InitialSolution(FS[2], FS[0], FS[1], FS[3]))
    assert np.array_equal(U, Oracle(raw=raw, order=2, freestream=FS).initial_solution())


def test_gmsh_roundtrip_and_reference_parser(tmp_path):
    raw = naca0012_ogrid(20, 10)
    path = str(tmp_path / "naca0012.msh")
    write_gmsh(raw, path)
    back = GmshParser.parse(path)
    assert np.array_equal(back.vertices, raw.vertices)
    assert [b.physical_name for b in back.edge_blocks] == ["Wall", "Farfield"]
    for a, b in zip(back.edge_blocks, raw.edge_blocks):
        assert np.array_equal(a.node_pairs, b.node_pairs)
    assert np.array_equal(back.element_blocks[0], raw.element_blocks[0])
    # the oracle's restatement of the reference parser reads the same mesh
    m = process_mesh(back, _fs_q(FS), 1.4)
    _check_mesh_equal(Oracle(msh_path=path, order=2, freestream=FS), m)


def test_gmsh_roundtrip_airfoil_blocks(tmp_path):
    """The reference's airfoil mesh (seven boundary line blocks, three "Wall" and four "Farfield")
    written as gmsh 4.1 and read back by the native reader: same vertices, blocks, names, triangles,
    and the same processed mesh as the oracle's own parser and process_mesh give for that file."""
    raw = airfoil_raw()
    path = str(tmp_path / "airfoil_rt.msh")
    write_gmsh(raw, path)
    back = GmshParser.parse(path)
    assert np.array_equal(back.vertices, raw.vertices)
    assert [b.physical_name for b in back.edge_blocks] == [b.physical_name for b in raw.edge_blocks]
    assert all(np.array_equal(a.node_pairs, b.node_pairs) for a, b in zip(back.edge_blocks, raw.edge_blocks))
    assert np.array_equal(back.element_blocks[0], raw.element_blocks[0])
    fs = (1.5, 0.8, 1.0, 100000.0)
    _check_mesh_equal(Oracle(msh_path=path, order=2, freestream=fs), process_mesh(back, _fs_q(fs), 1.4))


def test_gmsh_reader_line_endings_and_errors(tmp_path):
    """CRLF line ends and a last line without a newline read the same mesh (BufRead::lines drops
    one '\\r' before each '\\n'); where the reference's reader panics (no file, an entity without
    a physical name, a malformed number) DgmError DGM_BAD_ARG is raised."""
    raw = naca0012_ogrid(12, 6)
    path = tmp_path / "m.msh"
    write_gmsh(raw, str(path))
    txt = path.read_bytes()
    ref = GmshParser.parse(str(path))
    for name, data in (("crlf.msh", txt.replace(b"\n", b"\r\n")), ("nonl.msh", txt.rstrip(b"\n"))):
        (tmp_path / name).write_bytes(data)
        back = GmshParser.parse(str(tmp_path / name))
        assert np.array_equal(back.vertices, ref.vertices)
        assert all(np.array_equal(a.node_pairs, b.node_pairs) for a, b in zip(back.edge_blocks, ref.edge_blocks))
        assert np.array_equal(back.element_blocks[0], ref.element_blocks[0])
    lines = txt.decode().split("\n")
    i = lines.index("$PhysicalNames")
    bad_name = "\n".join(lines[:i + 2] + lines[i + 3:])          # drop the first physical name
    j = lines.index("$Nodes")
    k = next(n for n in range(j + 2, len(lines)) if len(lines[n].split()) == 3)  # first coordinate line
    bad_num = "\n".join(lines[:k] + ["1.0x " + " ".join(lines[k].split()[1:])] + lines[k + 1:])
    for name, data in (("noname.msh", bad_name), ("badnum.msh", bad_num)):
        (tmp_path / name).write_text(data)
        with pytest.raises(DgmError) as err:
            GmshParser.parse(str(tmp_path / name))
        assert err.value.status == 7
    with pytest.raises(DgmError) as err:
        GmshParser.parse(str(tmp_path / "missing.msh"))
    assert err.value.status == 7


def test_ogrid_geometry():
    raw = naca0012_ogrid(64, 32)
    m = process_mesh(raw, _fs_q(FS), 1.4)
    assert m.n_elements == 2 * 64 * 32
    assert m.n_edges == 64 * (3 * 32 + 1)
    assert len(m.boundary_element_indices) == 2 * 64
    r = np.hypot(raw.vertices[:, 0] - 0.5, raw.vertices[:, 1])
    assert abs(r.max() - 20.0) < 1e-12
    # colored numbering: every neighbour of an A triangle is a B triangle
    half = m.n_elements // 2
    nb = m.elem_neighbours
    a = nb[:half]
    assert ((a == -1) | (a >= half)).all()
    b = nb[half:]
    assert ((b == -1) | (b < half)).all()


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "dgm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dgm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol(built):
    from dgm_in_rust_b200 import _native
    lib = ctypes.CDLL(_native.library_path())
    syms = _header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert b"sm_100a" in _native.lib().dgm_version()


def test_library_built_for_sm100a(built):
    from dgm_in_rust_b200 import _native
    blob = open(_native.library_path(), "rb").read()
    assert b"sm_100a" in blob


def test_no_cpu_fallback_without_gpu(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    raw = naca0012_ogrid(8, 4)
    m = process_mesh(raw, _fs_q(FS), 1.4)
    with pytest.raises(DgmError) as ei:
        build_solver(m, 2, 1.4, 0.1, 1.0, 1)
    assert ei.value.status == 10  # DGM_NO_DEVICE


def test_status_strings_match_reference_messages(built):
    from dgm_in_rust_b200 import _native
    L = _native.lib()
    assert L.dgm_status_string(1) == b"Negative density found in HLLC!"
    assert L.dgm_status_string(2) == b"Negative pressure found in HLLC!"
    assert L.dgm_status_string(4) == b"Invalid number of boundary neighbours!"
    assert L.dgm_status_string(12) == b"Limiter worklist overflow"
