"""The .vtu writer (femgpu.vtk, the format of crates/io/src/vtk.rs): the
reference's own checks (UnstructuredGrid type, point count of unit_cube_tet(2),
named CellData, <?xml ... </VTKFile> framing) and a parse-back round trip of
points, cells and a solution field."""
import xml.etree.ElementTree as ET

import numpy as np

from femgpu import tet as T
from femgpu import vtk


def _parse(s):
    root = ET.fromstring(s)
    piece = root.find("UnstructuredGrid/Piece")
    arrays = {}
    for da in root.iter("DataArray"):
        arrays[da.get("Name") or "points"] = np.array(da.text.split(), dtype=np.float64)
    return root, piece, arrays


def test_tet_mesh_matches_reference_checks():
    coords, conn = T.unit_cube_tet(2)
    cells, ct = vtk.tet_cells(conn)
    s = vtk.vtu_string(coords, cells, ct, cell_data={"pressure": np.ones(len(conn))})
    assert s.startswith("<?xml") and s.endswith("</VTKFile>\n")
    assert 'type="UnstructuredGrid"' in s and f'NumberOfPoints="{len(coords)}"' in s
    assert 'Name="pressure"' in s and "<CellData>" in s
    root, piece, a = _parse(s)
    assert int(piece.get("NumberOfCells")) == len(conn)
    assert np.array_equal(a["connectivity"].reshape(-1, 4), conn)
    assert np.array_equal(a["types"], np.full(len(conn), vtk.VTK_TETRA))
    assert np.allclose(a["points"].reshape(-1, 3), coords, rtol=0, atol=1e-16)


def test_hex_lattice_roundtrip():
    nx, ny, nz, p = 3, 2, 4, 2
    pts = vtk.hex_lattice_points(nx, ny, nz, p)
    cells = vtk.hex_lattice_cells(nx, ny, nz, p)
    assert cells.shape == ((nx * p) * (ny * p) * (nz * p), 8)
    u = np.sin(np.pi * pts).prod(axis=1)
    s = vtk.vtu_string(pts, cells, vtk.VTK_HEXAHEDRON, point_data={"u": u})
    _, piece, a = _parse(s)
    assert int(piece.get("NumberOfPoints")) == len(pts)
    assert np.allclose(a["u"], u, rtol=1e-10, atol=1e-300)
    # every lattice hex has positive volume in VTK's vertex order
    P = pts[cells]
    vol = np.einsum("ij,ij->i", P[:, 1] - P[:, 0], np.cross(P[:, 3] - P[:, 0], P[:, 4] - P[:, 0]))
    assert np.all(vol > 0)


def test_quadratic_tet_order():
    coords, conn = T.unit_cube_tet(1)
    dofs, nd = T.p2_dofs(conn, len(coords))
    cells, ct = vtk.tet_cells(dofs)
    xyz = T.dof_coords(coords, dofs, nd)
    assert ct == vtk.VTK_QUADRATIC_TETRA
    # VTK edge nodes: midpoints of (0,1), (1,2), (0,2), (0,3), (1,3), (2,3)
    for c in cells:
        v = xyz[c[:4]]
        pairs = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]
        for k, (a, b) in enumerate(pairs):
            assert np.allclose(xyz[c[4 + k]], 0.5 * (v[a] + v[b]))
