"""Tetrahedral meshes and DOF maps for the tet PA operator (host side).

unit_cube_tet(n) builds the mesh of SimplexMesh::unit_cube_tet
(crates/mesh/src/simplex.rs:591-679): (n+1)^3 nodes numbered i fastest, each
sub-cube split into 6 tetrahedra around the diagonal v0 -> v6 in the order
[0,1,2,6], [0,2,3,6], [0,3,7,6], [0,7,4,6], [0,4,5,6], [0,5,1,6].

p2_dofs numbers the DOFs as DofManager::build_p2_tet does
(crates/space/src/dof_manager.rs:628-700): vertex DOFs are the node ids, and
each edge gets the next id at its first appearance in the element loop, with
the element's edges taken in the order (n0n1, n0n2, n0n3, n1n2, n1n3, n2n3).

p3_dofs numbers them as build_p3_tet (dof_manager.rs:484-600): each edge gets
two consecutive ids at its first appearance, the first near the smaller node
id; an element lists its edge pair in its own direction (near its first
vertex, then near its second); after all edges, each face (n0n1n2, n0n1n3,
n0n2n3, n1n2n3 per element) gets one id at its first appearance.
"""
from __future__ import annotations

import numpy as np

_CUBE_TETS = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])
_TET_EDGES = np.array([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]])


def unit_cube_tet(n):
    """(coords [(n+1)^3, 3], conn [6 n^3, 4] int32)."""
    np1 = n + 1
    k, j, i = np.meshgrid(np.arange(np1), np.arange(np1), np.arange(np1), indexing="ij")
    coords = np.stack([i / n, j / n, k / n], axis=-1).reshape(-1, 3).astype(np.float64)
    kk, jj, ii = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    kk, jj, ii = kk.ravel(), jj.ravel(), ii.ravel()

    def nid(a, b, c):
        return c * np1 * np1 + b * np1 + a

    v = np.stack([nid(ii, jj, kk), nid(ii + 1, jj, kk), nid(ii + 1, jj + 1, kk), nid(ii, jj + 1, kk),
                  nid(ii, jj, kk + 1), nid(ii + 1, jj, kk + 1), nid(ii + 1, jj + 1, kk + 1),
                  nid(ii, jj + 1, kk + 1)], axis=1)  # [cubes, 8], cubes in (k, j, i) loop order
    conn = v[:, _CUBE_TETS].reshape(-1, 4)          # 6 tets per cube, in cube order
    return coords, conn.astype(np.int32)


def p2_dofs(conn, n_nodes):
    """(elem_dofs [E, 10] int32, n_dofs): vertices, then edges numbered in
    order of first appearance."""
    E = conn.shape[0]
    a = conn[:, _TET_EDGES[:, 0]].astype(np.int64)
    b = conn[:, _TET_EDGES[:, 1]].astype(np.int64)
    key = np.minimum(a, b) * (n_nodes + 1) + np.maximum(a, b)  # [E, 6], row-major = loop order
    flat = key.ravel()
    uniq, first, inv = np.unique(flat, return_index=True, return_inverse=True)
    rank = np.empty(len(uniq), dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uniq))
    edge_dof = n_nodes + rank[inv].reshape(E, 6)
    dofs = np.concatenate([conn.astype(np.int64), edge_dof], axis=1)
    return dofs.astype(np.int32), int(n_nodes + len(uniq))


def _first_appearance_rank(keys):
    """rank of each key's first appearance in row-major order (0, 1, ...)"""
    flat = keys.ravel()
    uniq, first, inv = np.unique(flat, return_index=True, return_inverse=True)
    rank = np.empty(len(uniq), dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uniq))
    return rank[inv].reshape(keys.shape), len(uniq)


_TET_FACES = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])


def p3_dofs(conn, n_nodes):
    """(elem_dofs [E, 20] int32, n_dofs) in the numbering of build_p3_tet."""
    E = conn.shape[0]
    m = n_nodes + 1
    a = conn[:, _TET_EDGES[:, 0]].astype(np.int64)
    b = conn[:, _TET_EDGES[:, 1]].astype(np.int64)
    erank, n_edges = _first_appearance_rank(np.minimum(a, b) * m + np.maximum(a, b))
    d0 = n_nodes + 2 * erank          # near the smaller node id
    d1 = d0 + 1
    near_first = np.where(a < b, d0, d1)
    near_second = np.where(a < b, d1, d0)
    edges = np.stack([near_first, near_second], axis=2).reshape(E, 12)
    f = np.sort(conn[:, _TET_FACES].astype(np.int64), axis=2)  # [E, 4, 3]
    frank, n_faces = _first_appearance_rank((f[..., 0] * m + f[..., 1]) * m + f[..., 2])
    faces = n_nodes + 2 * n_edges + frank
    dofs = np.concatenate([conn.astype(np.int64), edges, faces], axis=1)
    return dofs.astype(np.int32), int(n_nodes + 2 * n_edges + n_faces)


def dof_coords(coords, elem_dofs, n_dofs):
    """Coordinates of every DOF (vertices, edge midpoints)."""
    out = np.zeros((n_dofs, 3))
    out[elem_dofs[:, :4].ravel()] = coords[elem_dofs[:, :4].ravel()]
    va = coords[elem_dofs[:, _TET_EDGES[:, 0]]]
    vb = coords[elem_dofs[:, _TET_EDGES[:, 1]]]
    if elem_dofs.shape[1] == 10:
        out[elem_dofs[:, 4:].ravel()] = (0.5 * (va + vb)).reshape(-1, 3)
    elif elem_dofs.shape[1] == 20:
        near = np.stack([(2 * va + vb) / 3, (va + 2 * vb) / 3], axis=2)  # [E, 6, 2, 3]
        out[elem_dofs[:, 4:16].ravel()] = near.reshape(-1, 3)
        cen = coords[elem_dofs[:, :4]][:, _TET_FACES].mean(axis=2)      # [E, 4, 3]
        out[elem_dofs[:, 16:].ravel()] = cen.reshape(-1, 3)
    return out


def unit_cube_boundary_mask(xyz, tol=1e-12):
    """Essential DOFs of all six faces of the unit cube (tags 1..6): on the
    Freudenthal mesh a DOF lies on a boundary face exactly when one of its
    coordinates is 0 or 1."""
    return (np.any((np.abs(xyz) < tol) | (np.abs(xyz - 1.0) < tol), axis=1)).astype(np.uint8)


def unit_cube_space(n, p):
    """coords, elem_dofs, n_dofs, essential mask of the order-p (1 to 3) space
    on unit_cube_tet(n)."""
    coords, conn = unit_cube_tet(n)
    if p == 1:
        dofs, nd = conn, coords.shape[0]
    elif p == 2:
        dofs, nd = p2_dofs(conn, coords.shape[0])
    elif p == 3:
        dofs, nd = p3_dofs(conn, coords.shape[0])
    else:
        raise ValueError("tet orders 1 to 3 are supported")
    mask = unit_cube_boundary_mask(dof_coords(coords, dofs, nd))
    return coords, dofs, nd, mask
