"""VTK XML unstructured-grid (.vtu) output of meshes and solution fields.

Mirrors the reference writer (crates/io/src/vtk.rs:140-240): an ASCII
<VTKFile type="UnstructuredGrid"> with Float64 points, Int32
connectivity / offsets, UInt8 cell types, then PointData and CellData arrays
(Float64, values written with 10 significant decimals as in write_data_array).

Cells:
  hex_lattice_cells: the DOF lattice of a structured hex space (any order) cut
    into linear hexahedra (VTK_HEXAHEDRON = 12), so every DOF is a point;
  tetrahedra: VTK_TETRA (10) from the 4 vertex nodes, or VTK_QUADRATIC_TETRA
    (24) from the 10 TetP2 DOFs, reordered from the DofManager edge order
    (01, 02, 03, 12, 13, 23) to VTK's (01, 12, 02, 03, 13, 23).
"""
from __future__ import annotations

import io

import numpy as np

VTK_TETRA, VTK_HEXAHEDRON, VTK_QUADRATIC_TETRA = 10, 12, 24
_P2_TO_VTK = np.array([0, 1, 2, 3, 4, 7, 5, 6, 8, 9])


def hex_lattice_points(nx, ny, nz, p, vcoord=None):
    """Coordinates of the DOF lattice (I fastest); trilinear map of the element
    vertices, or the unit cube when vcoord is None."""
    NI, NJ, NK = nx * p + 1, ny * p + 1, nz * p + 1
    k, j, i = np.meshgrid(np.arange(NK), np.arange(NJ), np.arange(NI), indexing="ij")
    if vcoord is None:
        return np.stack([i / (NI - 1), j / (NJ - 1), k / (NK - 1)], axis=-1).reshape(-1, 3)
    V = np.asarray(vcoord, dtype=np.float64).reshape(nz + 1, ny + 1, nx + 1, 3)
    ex, ey, ez = np.minimum(i // p, nx - 1), np.minimum(j // p, ny - 1), np.minimum(k // p, nz - 1)
    u, v, w = i / p - ex, j / p - ey, k / p - ez
    out = np.zeros(i.shape + (3,))
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                wt = (u if dx else 1 - u) * (v if dy else 1 - v) * (w if dz else 1 - w)
                out += wt[..., None] * V[ez + dz, ey + dy, ex + dx]
    return out.reshape(-1, 3)


def hex_lattice_cells(nx, ny, nz, p):
    """Linear hexahedra over the DOF lattice: [cells, 8] in VTK vertex order."""
    NI, NJ, NK = nx * p + 1, ny * p + 1, nz * p + 1
    k, j, i = np.meshgrid(np.arange(NK - 1), np.arange(NJ - 1), np.arange(NI - 1), indexing="ij")
    base = (k * NJ + j) * NI + i
    off = [0, 1, NI + 1, NI, NI * NJ, NI * NJ + 1, NI * NJ + NI + 1, NI * NJ + NI]
    return np.stack([base + o for o in off], axis=-1).reshape(-1, 8)


def tet_cells(elem_dofs):
    """(cells, vtk type) for TetP1 (4 nodes) or TetP2 (10 DOFs) element maps."""
    elem_dofs = np.asarray(elem_dofs)
    if elem_dofs.shape[1] == 4:
        return elem_dofs, VTK_TETRA
    return elem_dofs[:, _P2_TO_VTK], VTK_QUADRATIC_TETRA


def _rows(a, fmt):
    buf = io.StringIO()
    np.savetxt(buf, np.atleast_2d(a), fmt=fmt, delimiter=" ")
    return "".join("          " + line + "\n" for line in buf.getvalue().splitlines())


def _array(name, values, ncomp):
    values = np.asarray(values, dtype=np.float64).reshape(-1, ncomp)
    return (f'        <DataArray type="Float64" Name="{name}" NumberOfComponents="{ncomp}" format="ascii">\n'
            + _rows(values, "%.10e") + "        </DataArray>\n")


def vtu_string(points, cells, cell_type, point_data=None, cell_data=None):
    """The .vtu document as a string.  point_data / cell_data: {name: array}
    (scalars, or [n, k] vectors)."""
    points = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    cells = np.asarray(cells, dtype=np.int64)
    n_pts, n_cells, npe = points.shape[0], cells.shape[0], cells.shape[1]
    s = ['<?xml version="1.0"?>\n',
         '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n',
         '  <UnstructuredGrid>\n',
         f'    <Piece NumberOfPoints="{n_pts}" NumberOfCells="{n_cells}">\n',
         '      <Points>\n',
         '        <DataArray type="Float64" NumberOfComponents="3" format="ascii">\n',
         _rows(points, "%.17g"),
         '        </DataArray>\n', '      </Points>\n', '      <Cells>\n',
         '        <DataArray type="Int32" Name="connectivity" format="ascii">\n',
         _rows(cells, "%d"), '        </DataArray>\n',
         '        <DataArray type="Int32" Name="offsets" format="ascii">\n',
         _rows(np.arange(1, n_cells + 1) * npe, "%d"), '        </DataArray>\n',
         '        <DataArray type="UInt8" Name="types" format="ascii">\n',
         _rows(np.full(n_cells, cell_type), "%d"), '        </DataArray>\n', '      </Cells>\n']
    for tag, data in (("PointData", point_data), ("CellData", cell_data)):
        if data:
            s.append(f"      <{tag}>\n")
            for name, val in data.items():
                val = np.asarray(val)
                s.append(_array(name, val, 1 if val.ndim == 1 else val.shape[-1]))
            s.append(f"      </{tag}>\n")
    s += ["    </Piece>\n", "  </UnstructuredGrid>\n", "</VTKFile>\n"]
    return "".join(s)


def write_vtu(path, points, cells, cell_type, point_data=None, cell_data=None):
    with open(path, "w") as f:
        f.write(vtu_string(points, cells, cell_type, point_data, cell_data))


def write_hex_solution(path, nx, ny, nz, p, u, name="u", vcoord=None):
    """A structured hex space's DOF vector (plain layout) on its DOF lattice."""
    write_vtu(path, hex_lattice_points(nx, ny, nz, p, vcoord), hex_lattice_cells(nx, ny, nz, p),
              VTK_HEXAHEDRON, point_data={name: np.asarray(u)})
