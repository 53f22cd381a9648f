"""Tetrahedral meshes: boundary faces, ground surface, point location and P1 templates.

Restates adtlert/mesh/core3d.py:16-230 (``Mesh3D``) and adtlert/fem/tetrahedron.py:37-56
(``build_tetrahedron_p1_data``) in float64 NumPy. This is host set-up, run once per operator.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import _as_numpy

# local vertex triples of the four faces of a tetrahedron (core3d.py:16)
TETRA_FACES = ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1))


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
