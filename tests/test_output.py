"""Result output in the reference's VTK format (src/io/write_results.rs:8-93).

CPU: the text layout against the reference's own output file structure (a legacy ASCII file of
vtkio: empty title, one-line data blocks, one cell type per line, empty POINT_DATA) and Rust's
f64 formatting.  GPU: the device cell fields against the reference's expressions evaluated in
numpy on the downloaded state (bitwise), and a written file read back.
"""
import os

import numpy as np
import pytest

from conftest import airfoil_raw
from dgm_in_rust_b200 import InitialSolution, build_solver, freestream_quantity, naca0012_ogrid, process_mesh
from dgm_in_rust_b200.output import format_f64, solution_path, vtk_text, write_to_vtk


def test_rust_f64_display():
    cases = [(1.0, "1"), (-20.0, "-20"), (0.141414, "0.141414"),
             (9.833257050678418e-18, "0.000000000000000009833257050678418"), (1e20, "100000000000000000000"),
             (0.1 + 0.2, "0.30000000000000004"), (float("nan"), "NaN"), (float("inf"), "inf"), (-0.0, "-0"),
             (0.0, "0")]
    for x, s in cases:
        assert format_f64(x) == s, (x, format_f64(x))


def test_vtk_layout_matches_reference_structure():
    v = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]])
    t = np.array([[0, 1, 2], [1, 3, 2]])
    f = np.array([[1.0, 0.5, 0.0, 0.7142857142857143], [1.25, -0.5, 0.25, 1.0]])
    lines = vtk_text(v, t, f).split("\n")
    assert lines[:6] == ["# vtk DataFile Version 2.0", "", "ASCII", "", "DATASET UNSTRUCTURED_GRID", "POINTS 4 double"]
    assert lines[6] == "0 0 0 1 0 0 0 1 0 1 1 0"
    assert lines[7:12] == ["", "CELLS 2 8", "3 0 1 2 3 1 3 2", "", "CELL_TYPES 2"]
    assert lines[12:14] == ["5", "5"]
    assert lines[14:20] == ["", "", "POINT_DATA 4", "", "CELL_DATA 2", ""]
    assert lines[20:23] == ["SCALARS Density double 1", "LOOKUP_TABLE default", "1 1.25"]
    assert lines[23:26] == ["", "VECTORS Velocity double", "0.5 0 0 -0.5 0.25 0"]
    assert lines[26:30] == ["", "SCALARS Pressure double 1", "LOOKUP_TABLE default", "0.7142857142857143 1"]
    assert lines[30:] == ["", ""]


def test_section_sizes_on_the_reference_mesh(tmp_path):
    raw = airfoil_raw()
    mesh = process_mesh(raw, freestream_quantity(0.8, 1.5, 1.0, 1e5, 1.4), 1.4)
    ne, nv = mesh.n_elements, mesh.vertices.shape[0]
    path = write_to_vtk(solution_path(20, str(tmp_path / "outputfiles" / "solutions")), mesh, np.ones((ne, 4)))
    assert path.endswith(os.path.join("solutions", "step=20.vtk"))
    lines = open(path).read().split("\n")
    # the reference's outputfiles/mesh.vtk for this mesh: POINTS 1961, CELLS 3738 14952, 5883 point
    # values and 14952 cell entries on one line each, POINT_DATA 1961, CELL_DATA 3738
    assert (nv, ne) == (1961, 3738)
    assert lines[5] == "POINTS 1961 double" and len(lines[6].split()) == 5883
    assert lines[8] == "CELLS 3738 14952" and len(lines[9].split()) == 14952
    assert lines[11] == "CELL_TYPES 3738" and lines[12:12 + ne] == ["5"] * ne
    assert lines[12 + ne + 2] == "POINT_DATA 1961" and lines[12 + ne + 4] == "CELL_DATA 3738"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_cell_fields_match_reference_expressions(built, tmp_path, precision):
    raw = naca0012_ogrid(32, 16)
    mesh = process_mesh(raw, freestream_quantity(0.8, 1.25, 1.0, 1.0 / 1.4, 1.4), 1.4)
    s = build_solver(mesh, 2, 1.4, 0.1, 1.0e30, 6, precision=precision)
    td, sd = s.temporal_disc, s.spatial_disc
    td.set_initial_on_device(InitialSolution(1.0, 1.25, 0.8, 1.0 / 1.4))
    td.advance(6)
    td.synchronize()
    U = sd.new_state()
    td.download(U)
    f = sd.cell_fields()
    rho, mx, my, en = U[:, 0, 0], U[:, 1, 0], U[:, 2, 0], U[:, 3, 0]
    u, v = mx / rho, my / rho
    p = (1.4 - 1.0) * (en - 0.5 * rho * (u * u + v * v))
    assert np.array_equal(f, np.stack([rho, u, v, p], axis=1))
    path = s.write_results(str(tmp_path / "solutions"))
    assert path.endswith("step=6.vtk")
    lines = open(path).read().split("\n")
    k = lines.index("SCALARS Density double 1")
    assert np.array_equal(np.array([float(x) for x in lines[k + 2].split()]), rho)
    s.close()


def test_native_writer_matches_layout_bytes(tmp_path):
    """The library's writer (dgm_vtk_write) produces exactly the text vtk_text lays out, for
    magnitudes from 1e-30 to 1e30 and the special values Rust prints as NaN, inf, -inf, -0."""
    from dgm_in_rust_b200 import freestream_quantity, naca0012_ogrid, process_mesh
    from dgm_in_rust_b200.output import vtk_text, write_to_vtk
    rng = np.random.default_rng(1)
    m = process_mesh(naca0012_ogrid(32, 16), freestream_quantity(0.8, 1.25, 1.0, 1 / 1.4, 1.4), 1.4)
    f = rng.standard_normal((m.n_elements, 4)) * 10.0 ** rng.integers(-30, 30, (m.n_elements, 4))
    specials = [np.nan, np.inf, -np.inf, -0.0, 0.0, 5e-324, 1.7976931348623157e308, 1.0, 0.1, 2.5e20, 1e-7]
    f.reshape(-1)[:len(specials)] = specials
    path = write_to_vtk(str(tmp_path / "solutions" / "step=3.vtk"), m, f)
    with open(path) as fh:
        assert fh.read() == vtk_text(m.vertices, m.elem_vertices, f)


def _reference_airfoil_path(tmp_path):
    """The reference's own input fixture (inputfiles/airfoil.msh), unpacked from tests/golden."""
    import gzip
    from conftest import GOLDEN
    path = tmp_path / "airfoil.msh"
    path.write_bytes(gzip.open(os.path.join(GOLDEN, "reference_airfoil.msh.gz")).read())
    return str(path)


def test_reference_output_file_reproduced_byte_for_byte(tmp_path):
    """Pinned to an output the reference itself produced: outputfiles/mesh.vtk of DGM_in_rust, the
    VTK file its write_to_vtk (src/io/write_results.rs:8-93) wrote for inputfiles/airfoil.msh
    with NaN cell fields.  The reference's airfoil.msh goes through the native gmsh reader
    (mesh_parser.rs:28-158) and process_mesh; the file written by the native writer and the text of
    the layout restatement both equal the reference's file byte for byte (209,182 bytes: vertex
    order and coordinates, triangle order, Rust's f64 formatting of every number and of NaN)."""
    import gzip
    from conftest import GOLDEN
    from dgm_in_rust_b200 import GmshParser
    ref = gzip.open(os.path.join(GOLDEN, "reference_mesh.vtk.gz")).read()
    raw = GmshParser.parse(_reference_airfoil_path(tmp_path))
    mesh = process_mesh(raw, freestream_quantity(0.8, 1.5, 1.0, 1e5, 1.4), 1.4)
    fields = np.full((mesh.n_elements, 4), np.nan)
    path = write_to_vtk(str(tmp_path / "solutions" / "mesh.vtk"), mesh, fields)
    with open(path, "rb") as fh:
        native = fh.read()
    assert len(native) == len(ref) == 209182
    assert native == ref
    assert vtk_text(mesh.vertices, mesh.elem_vertices, fields).encode() == ref


def test_airfoil_fixture_arrays_match_reference_file(tmp_path):
    """The stored arrays of the reference's airfoil mesh (airfoil_mesh.npz, used by the parity
    tests) are what the native reader gives for the reference's airfoil.msh."""
    from dgm_in_rust_b200 import GmshParser
    raw = GmshParser.parse(_reference_airfoil_path(tmp_path))
    stored = airfoil_raw()
    assert np.array_equal(raw.vertices, stored.vertices)
    assert [b.physical_name for b in raw.edge_blocks] == [b.physical_name for b in stored.edge_blocks]
    for a, b in zip(raw.edge_blocks, stored.edge_blocks):
        assert np.array_equal(a.node_pairs, b.node_pairs)
    assert len(raw.element_blocks) == len(stored.element_blocks)
    for a, b in zip(raw.element_blocks, stored.element_blocks):
        assert np.array_equal(a, b)
