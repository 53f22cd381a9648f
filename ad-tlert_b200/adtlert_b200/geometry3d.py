"""Tetrahedral meshes: boundary faces, ground surface, point location, P1 and P2 templates.

Restates adtlert/mesh/core3d.py:16-234 (``Mesh3D``, ``build_quadratic_topology``) and
adtlert/fem/tetrahedron.py:37-127 (P1 and ten-node P2 tetrahedron data) in float64 NumPy. This
is host set-up, run once per operator.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import _as_numpy

# local vertex triples of the four faces of a tetrahedron (core3d.py:16)
TETRA_FACES = ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1))
# edges of the ten-node tetrahedron after its four vertices, and of the six-node face after its
# three (the dof order of tetrahedron.py:13 and core3d.py:211-234)
P2_CELL_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))
P2_FACE_EDGES = ((0, 1), (1, 2), (2, 0))


def _edge_matrices(cell_nodes: np.ndarray) -> np.ndarray:
    return np.stack([cell_nodes[:, i] - cell_nodes[:, 0] for i in (1, 2, 3)], axis=-1)


def tetrahedron_volumes(nodes: np.ndarray, cells: np.ndarray) -> np.ndarray:
    return np.abs(np.linalg.det(_edge_matrices(nodes[cells]))) / 6.0


def boundary_topology(cells: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Faces that belong to one cell only (vertex ids sorted, rows sorted) and their cells
    (core3d.py:39-47)."""

    faces = np.sort(cells[:, TETRA_FACES], axis=-1).reshape(-1, 3)
    unique, first, counts = np.unique(faces, axis=0, return_index=True, return_counts=True)
    keep = counts == 1
    return unique[keep].astype(np.int32), (first[keep] // 4).astype(np.int32)


def boundary_geometry(nodes, cells, faces, face_cells):
    """Centers, areas and outward unit normals of boundary faces (core3d.py:50-65)."""

    face_nodes = nodes[faces]
    centers = face_nodes.mean(axis=1)
    cross = np.cross(face_nodes[:, 1] - face_nodes[:, 0], face_nodes[:, 2] - face_nodes[:, 0])
    norm = np.linalg.norm(cross, axis=1)
    normals = cross / norm[:, None]
    outward = np.sum(normals * (centers - nodes[cells[face_cells]].mean(axis=1)), axis=1) >= 0.0
    return centers, 0.5 * norm, normals * np.where(outward, 1.0, -1.0)[:, None]


def locate_points_in_tetrahedra(nodes, cells, points, tol: float = 1e-8) -> tuple[np.ndarray, np.ndarray]:
    """Containing cell and barycentric weights of every point (core3d.py:68-107): the cells
    around a coincident node first, otherwise every cell whose padded bounding box holds it."""

    nodes, cells = np.asarray(nodes, dtype=float), np.asarray(cells, dtype=np.int64)
    points = np.asarray(points, dtype=float)
    cell_nodes = nodes[cells]
    origins = cell_nodes[:, 0]
    inverse = np.linalg.inv(_edge_matrices(cell_nodes))
    lower, upper = cell_nodes.min(axis=1) - tol, cell_nodes.max(axis=1) + tol
    ids = np.full(points.shape[0], -1, dtype=np.int64)
    weights = np.zeros((points.shape[0], 4))
    for p, point in enumerate(points):
        nearest = int(np.argmin(np.linalg.norm(nodes - point, axis=1)))
        if np.linalg.norm(nodes[nearest] - point) <= tol:
            candidates = np.flatnonzero(np.any(cells == nearest, axis=1))
        else:
            candidates = np.flatnonzero(np.all((point >= lower) & (point <= upper), axis=1))
        for c in candidates:
            local = inverse[c] @ (point - origins[c])
            bary = np.asarray((1.0 - local.sum(), *local))
            if np.all(bary >= -tol) and np.all(bary <= 1.0 + tol):
                bary[np.abs(bary) <= tol] = 0.0
                ids[p], weights[p] = c, bary / bary.sum()
                break
    if np.any(ids < 0):
        raise ValueError(f"points lie outside the tetrahedral mesh: indices={np.flatnonzero(ids < 0).tolist()}")
    return ids, weights


def tetrahedron_stiffness(nodes: np.ndarray, cells: np.ndarray) -> np.ndarray:
    """Unit-conductivity P1 stiffness templates ``|T| G G^T`` (tetrahedron.py:37-56)."""

    jac = _edge_matrices(nodes[cells])
    reference = np.asarray(((-1.0, -1.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)))
    gradients = np.einsum("ij,ejk->eik", reference, np.linalg.inv(jac))
    volumes = np.abs(np.linalg.det(jac)) / 6.0
    return volumes[:, None, None] * np.einsum("eid,ejd->eij", gradients, gradients)


def quadratic_topology(nodes: np.ndarray, cells: np.ndarray, faces: np.ndarray):
    """P2 dofs shared between cells: the vertices keep their numbers and every edge midpoint is
    numbered once, in the order the cells first use it (cell by cell, edges 01, 12, 20, 03, 13,
    23), as core3d.py:211-234 numbers them. Returns the dof coordinates, the cell dofs (C x 10:
    vertices, then edge midpoints) and the face dofs (F x 6: vertices, then edges 01, 12, 20)."""

    nodes = np.asarray(nodes, dtype=float)
    cells = np.asarray(cells, dtype=np.int64)
    faces = np.asarray(faces, dtype=np.int64)
    n = len(nodes)
    pairs = np.stack([cells[:, [i, j]] for i, j in P2_CELL_EDGES], axis=1).reshape(-1, 2)
    lo, hi = pairs.min(axis=1), pairs.max(axis=1)
    keys = lo * n + hi
    unique, first, inverse = np.unique(keys, return_index=True, return_inverse=True)
    rank = np.empty(len(unique), dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(unique))
    cell_mid = (n + rank[inverse]).reshape(-1, 6)
    order = np.argsort(rank)
    ua, ub = unique[order] // n, unique[order] % n
    dof_nodes = np.vstack((nodes, 0.5 * (nodes[ua] + nodes[ub])))
    face_pairs = np.stack([faces[:, [i, j]] for i, j in P2_FACE_EDGES], axis=1).reshape(-1, 2)
    face_keys = face_pairs.min(axis=1) * n + face_pairs.max(axis=1)
    position = np.searchsorted(unique, face_keys)
    if np.any(position >= len(unique)) or np.any(unique[np.minimum(position, len(unique) - 1)] != face_keys):
        raise ValueError("a boundary face edge is not an edge of any cell")
    face_mid = (n + rank[position]).reshape(-1, 3)
    return dof_nodes, np.hstack((cells, cell_mid)), np.hstack((faces, face_mid))


def p2_shape_values(barycentric: np.ndarray) -> np.ndarray:
    """Ten-node tetrahedron shape functions at barycentric points: l_i (2 l_i - 1) at the
    vertices, 4 l_i l_j at the edges (tetrahedron.py:59-66)."""

    b = np.asarray(barycentric, dtype=float)
    edges = np.stack([4.0 * b[..., i] * b[..., j] for i, j in P2_CELL_EDGES], axis=-1)
    return np.concatenate((b * (2.0 * b - 1.0), edges), axis=-1)


def tetrahedron_p2_stiffness(nodes: np.ndarray, cells: np.ndarray) -> np.ndarray:
    """Unit-conductivity ten-node stiffness templates (tetrahedron.py:92-127). The shape-function
    gradients are linear, so the 4-point symmetric rule (barycentric points with one coordinate
    (5 + 3 sqrt 5) / 20 and three (5 - sqrt 5) / 20, weights |T| / 4) integrates G G^T exactly;
    gradients: (4 l_i - 1) grad l_i at vertex i, 4 (l_i grad l_j + l_j grad l_i) at edge ij."""

    jac = _edge_matrices(nodes[cells])
    reference = np.asarray(((-1.0, -1.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)))
    grad = np.einsum("ij,ejk->eik", reference, np.linalg.inv(jac))  # (C, 4, 3) of the l_i
    volumes = np.abs(np.linalg.det(jac)) / 6.0
    major, minor = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0, (5.0 - np.sqrt(5.0)) / 20.0
    stiffness = np.zeros((len(cells), 10, 10))
    for q in range(4):
        lam = np.full(4, minor)
        lam[q] = major
        g = np.concatenate((
            (4.0 * lam - 1.0)[None, :, None] * grad,
            np.stack([4.0 * (lam[i] * grad[:, j] + lam[j] * grad[:, i]) for i, j in P2_CELL_EDGES], axis=1),
        ), axis=1)
        stiffness += np.einsum("eid,ejd->eij", g, g)
    return stiffness * (volumes / 4.0)[:, None, None]


def p2_triangle_mass(area: float) -> np.ndarray:
    """Six-node triangle mass matrix (vertices, then edges 01, 12, 20), exact: area / 180 times
    6 / -1 between vertices, 32 / 16 between edge midpoints, -4 between a vertex and the midpoint
    of the opposite edge, 0 otherwise (the matrix tetrahedron.py:69-89 integrates with a
    degree-4 rule)."""

    m = np.asarray((
        (6, -1, -1, 0, -4, 0),
        (-1, 6, -1, 0, 0, -4),
        (-1, -1, 6, -4, 0, 0),
        (0, 0, -4, 32, 16, 16),
        (-4, 0, 0, 16, 32, 16),
        (0, -4, 0, 16, 16, 32),
    ), dtype=float)
    return float(area) / 180.0 * m


@dataclass(frozen=True)
class Mesh3D:
    """Four-node tetrahedral mesh with boundary-face metadata (float64 host arrays)."""

    nodes: np.ndarray
    cells: np.ndarray
    boundary_faces: np.ndarray
    boundary_face_cells: np.ndarray
    boundary_face_centers: np.ndarray
    boundary_face_areas: np.ndarray
    boundary_face_normals: np.ndarray
    surface_face_mask: np.ndarray
    surface_reference_level: float
    flat_surface: bool
    cell_volumes: np.ndarray

    @classmethod
    def from_arrays(cls, nodes, cells, *, surface_face_mask=None) -> Mesh3D:
        """Validate and index a tetrahedral mesh; the ground surface defaults to the
        upward-facing exterior faces (core3d.py:124-178)."""

        nodes = _as_numpy(nodes, float)
        cells = _as_numpy(cells, np.int64)
        if nodes.ndim != 2 or nodes.shape[1] != 3:
            raise ValueError("3D nodes must have shape (num_nodes, 3)")
        if cells.ndim != 2 or cells.shape[1] != 4:
            raise ValueError("3D cells must have shape (num_cells, 4)")
        if cells.size == 0:
            raise ValueError("tetrahedral mesh must contain at least one cell")
        if np.any(cells < 0) or np.any(cells >= nodes.shape[0]):
            raise ValueError("cells reference nodes outside the mesh")
        used = np.unique(cells)
        if used.size != nodes.shape[0]:
            remap = np.full(nodes.shape[0], -1, dtype=np.int64)
            remap[used] = np.arange(used.size)
            nodes, cells = nodes[used], remap[cells]
        volumes = tetrahedron_volumes(nodes, cells)
        if np.any(volumes <= 0.0):
            raise ValueError("cells must define non-degenerate tetrahedra")
        faces, face_cells = boundary_topology(cells)
        centers, areas, normals = boundary_geometry(nodes, cells, faces, face_cells)
        if surface_face_mask is None:
            surface = normals[:, 2] > 1e-8
        else:
            surface = _as_numpy(surface_face_mask, bool).reshape(-1)
            if surface.shape != (faces.shape[0],):
                raise ValueError(
                    f"surface_face_mask must have one entry per boundary face ({surface.shape} != ({faces.shape[0]},))"
                )
        if not np.any(surface):
            raise ValueError("could not identify any upward-facing terrain surface faces")
        surface_nodes = np.unique(faces[surface])
        tol = max(1e-8, max(float(np.ptp(nodes[:, 2])), 1.0) * 1e-8)
        return cls(
            nodes=nodes,
            cells=cells.astype(np.int32),
            boundary_faces=faces,
            boundary_face_cells=face_cells,
            boundary_face_centers=centers,
            boundary_face_areas=areas,
            boundary_face_normals=normals,
            surface_face_mask=surface,
            surface_reference_level=float(np.max(nodes[:, 2])),
            flat_surface=bool(np.ptp(nodes[surface_nodes, 2]) <= tol),
            cell_volumes=volumes,
        )

    @property
    def node_count(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def cell_count(self) -> int:
        return int(self.cells.shape[0])

    @property
    def dimension(self) -> int:
        return 3

    @property
    def is_flat_surface(self) -> bool:
        return bool(self.flat_surface)

    def locate_points(self, points, tol: float = 1e-8) -> tuple[np.ndarray, np.ndarray]:
        return locate_points_in_tetrahedra(self.nodes, self.cells, points, tol=tol)
