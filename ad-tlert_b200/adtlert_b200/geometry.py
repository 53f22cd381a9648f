"""2D meshes and ABMN surveys with the metadata the 2.5D operator needs, plus the mesh
operations of the terrain discretizations (H2 refinement, columnar expansion, P2 topology).

``Mesh.from_arrays`` / ``Survey.from_arrays`` mirror the reference constructors
(adtlert/mesh/core.py:576-630, adtlert/survey/core.py:34-61): same validation, same boundary
and surface metadata, computed here with vectorized NumPy/SciPy. The operators also accept the
reference's own ``Mesh``/``Survey`` objects (anything exposing ``nodes``, ``cells`` and
``electrode_positions``/``measurements``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import dijkstra

REMOTE_ELECTRODE = -1


def _as_numpy(value, dtype=None) -> np.ndarray:
    if hasattr(value, "detach"):
        value = value.detach().cpu().numpy()
    return np.asarray(value, dtype=dtype)


def cell_edges(cells: np.ndarray) -> np.ndarray:
    """``(cells, width, 2)`` node pairs (sorted) of every polygon edge."""

    return np.sort(np.stack((cells, np.roll(cells, -1, axis=1)), axis=-1), axis=-1)


def boundary_edges_of(cells: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Boundary edges (sorted pairs, lexicographic order) and the first cell owning each."""

    flat = cell_edges(cells).reshape(-1, 2)
    edges, first, counts = np.unique(flat, axis=0, return_index=True, return_counts=True)
    keep = counts == 1
    return edges[keep], first[keep] // cells.shape[1]


def top_surface_path(nodes: np.ndarray, edges: np.ndarray, tol: float = 1e-8) -> np.ndarray:
    """Ordered top-surface node path between the upper-left and upper-right boundary corners.

    Shortest path over boundary edges whose cost grows with depth below the highest boundary
    edge (length * (1 + 100 * depth / span)), as adtlert/mesh/core.py:124-174 defines it.
    """

    boundary = np.unique(edges)
    x = nodes[boundary, 0]

    def corner(extreme: float) -> int:
        candidates = boundary[np.abs(x - extreme) <= tol]
        order = np.lexsort((nodes[candidates, 0], -nodes[candidates, 1]))
        return int(candidates[order[0]])

    start, stop = corner(float(x.min())), corner(float(x.max()))
    if start == stop:
        return np.asarray([start])
    centers_y = nodes[edges].mean(axis=1)[:, 1]
    lengths = np.linalg.norm(nodes[edges[:, 1]] - nodes[edges[:, 0]], axis=1)
    span = max(float(centers_y.max() - centers_y.min()), tol)
    cost = lengths * (1.0 + 100.0 * (centers_y.max() - centers_y) / span)
    n = nodes.shape[0]
    graph = sp.coo_matrix(
        (np.concatenate((cost, cost)), (np.concatenate((edges[:, 0], edges[:, 1])), np.concatenate((edges[:, 1], edges[:, 0])))),
        shape=(n, n),
    ).tocsr()
    _, predecessors = dijkstra(graph, directed=False, indices=start, return_predecessors=True)
    if predecessors[stop] < 0:
        return np.asarray([start, stop])
    path = [stop]
    while path[-1] != start:
        path.append(int(predecessors[path[-1]]))
    return np.asarray(path[::-1])


@dataclass(frozen=True)
class Mesh:
    """2D triangle or quadrilateral mesh with boundary and surface metadata (float64 geometry)."""

    nodes: np.ndarray
    cells: np.ndarray
    boundary_edges: np.ndarray
    boundary_edge_cells: np.ndarray
    boundary_edge_centers: np.ndarray
    boundary_edge_lengths: np.ndarray
    boundary_edge_normals: np.ndarray
    surface_node_ids: np.ndarray
    surface_edge_mask: np.ndarray
    surface_reference_level: float
    flat_surface: bool
    cell_areas: np.ndarray

    @classmethod
    def from_arrays(cls, nodes, cells, *, surface_node_ids=None) -> Mesh:
        nodes = _as_numpy(nodes, float)
        cells = _as_numpy(cells, np.int64)
        surface = None if surface_node_ids is None else _as_numpy(surface_node_ids, np.int64)
        if nodes.ndim != 2 or nodes.shape[1] != 2:
            raise ValueError("nodes must have shape (num_nodes, 2)")
        if cells.ndim != 2 or cells.shape[1] not in (3, 4):
            raise ValueError("cells must have shape (num_cells, 3) or (num_cells, 4)")
        if np.any(cells < 0):
            raise ValueError("cells contain negative node indices")
        if cells.size and np.any(cells >= nodes.shape[0]):
            raise ValueError("cells reference nodes outside the mesh")
        used = np.unique(cells)
        if used.size != nodes.shape[0]:
            remap = np.full(nodes.shape[0], -1, dtype=np.int64)
            remap[used] = np.arange(used.size)
            nodes, cells = nodes[used], remap[cells]
            surface = None if surface is None else remap[surface]
        xy = nodes[cells]
        areas = 0.5 * np.abs(np.sum(xy[..., 0] * np.roll(xy[..., 1], -1, 1) - np.roll(xy[..., 0], -1, 1) * xy[..., 1], axis=1))
        if np.any(areas <= 0.0):
            raise ValueError("cells must define non-degenerate 2D polygons")
        edges, edge_cells = boundary_edges_of(cells)
        ends = nodes[edges]
        centers = ends.mean(axis=1)
        vectors = ends[:, 1] - ends[:, 0]
        lengths = np.linalg.norm(vectors, axis=1)
        normals = np.stack((vectors[:, 1], -vectors[:, 0]), axis=1) / lengths[:, None]
        inside = nodes[cells[edge_cells]].mean(axis=1)
        normals *= np.where(np.sum(normals * (centers - inside), axis=1) >= 0.0, 1.0, -1.0)[:, None]
        path = top_surface_path(nodes, edges) if surface is None else surface
        pairs = np.sort(np.stack((path[:-1], path[1:]), axis=1), axis=1)
        key = edges[:, 0] * nodes.shape[0] + edges[:, 1]
        mask = np.isin(key, pairs[:, 0] * nodes.shape[0] + pairs[:, 1])
        top = nodes[path]
        flat = bool(top.size == 0 or np.max(np.abs(top[:, 1] - top[0, 1])) <= 1e-8)
        level = float(top[:, 1].mean()) if top.size else 0.0
        return cls(nodes, cells, edges, edge_cells, centers, lengths, normals, path, mask, level, flat, areas)

    @property
    def node_count(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def cell_count(self) -> int:
        return int(self.cells.shape[0])

    @property
    def is_flat_surface(self) -> bool:
        return bool(self.flat_surface)

    @property
    def cell_node_count(self) -> int:
        return int(self.cells.shape[1])

    @property
    def is_triangle_mesh(self) -> bool:
        return self.cell_node_count == 3

    @property
    def is_quadrilateral_mesh(self) -> bool:
        return self.cell_node_count == 4

    @property
    def surface_nodes(self) -> np.ndarray:
        return self.nodes[self.surface_node_ids]

    def locate_points(self, points, tol: float = 1e-4) -> tuple[np.ndarray, np.ndarray]:
        return locate_points(self.nodes, self.cells, _as_numpy(points, float), tol)

    def _require_triangles(self, operation: str) -> None:
        if not self.is_triangle_mesh:
            raise ValueError(f"{operation} is currently implemented for triangle meshes only")

    def refine_uniform(self) -> tuple[Mesh, np.ndarray]:
        """Split every triangle into four through its edge midpoints (H2); returns the refined
        mesh and the parent cell of each child (adtlert/mesh/core.py:326-337, 689-698)."""

        self._require_triangles("uniform refinement")
        c = self.cells
        surface = self.surface_node_ids
        pairs = np.concatenate((c[:, [0, 1, 1, 2, 2, 0]].reshape(-1, 2),
                                np.stack((surface[:-1], surface[1:]), axis=1)))
        points, ids = midpoint_nodes(self.nodes, pairs)
        m01, m12, m20 = ids[:3 * len(c)].reshape(-1, 3).T
        n0, n1, n2 = c.T
        cells = np.stack((np.stack((n0, m01, m20), 1), np.stack((n1, m12, m01), 1), np.stack((n2, m20, m12), 1),
                          np.stack((m01, m12, m20), 1)), axis=1).reshape(-1, 3)
        refined_surface = np.empty(max(2 * len(surface) - 1, 0), dtype=np.int64)
        refined_surface[0::2], refined_surface[1::2] = surface, ids[3 * len(c):]
        refined = Mesh.from_arrays(points, cells, surface_node_ids=refined_surface)
        return refined, np.repeat(np.arange(len(c), dtype=np.int64), 4)

    def expand_columnar_cells(self, tol: float = 1e-6) -> tuple[Mesh, np.ndarray] | None:
        """Complete single-triangle terrain strips into triangulated quads, or ``None`` when the
        mesh is not such a structure (adtlert/mesh/core.py:466-540, 723-736)."""

        if not self.is_triangle_mesh:
            return None
        expanded = expand_columnar_triangles(self.nodes, self.cells, tol)
        if expanded is None:
            return None
        nodes, cells, parents = expanded
        return Mesh.from_arrays(nodes, cells, surface_node_ids=self.surface_node_ids), parents

    def build_quadratic_topology(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Shared-edge P2 nodes, cells ``(v0, v1, v2, m01, m12, m20)`` and boundary edges
        ``(a, b, m_ab)`` (adtlert/mesh/core.py:543-555, 738-744)."""

        self._require_triangles("quadratic topology")
        c, boundary = self.cells, self.boundary_edges
        pairs = np.concatenate((c[:, [0, 1, 1, 2, 2, 0]].reshape(-1, 2), boundary))
        points, ids = midpoint_nodes(self.nodes, pairs)
        cells = np.hstack((c, ids[:3 * len(c)].reshape(-1, 3)))
        return points, cells, np.column_stack((boundary, ids[3 * len(c):]))


def first_use_numbers(keys: np.ndarray, start: int) -> tuple[np.ndarray, np.ndarray]:
    """Number the distinct values of a key sequence ``start, start + 1, ...`` in the order of
    their first occurrence. Returns each key's number and, per number, the position of its first
    occurrence (the sequence the reference's incremental node builders produce)."""

    unique, first, inverse = np.unique(np.asarray(keys, dtype=np.int64), return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty(len(unique), dtype=np.int64)
    rank[order] = np.arange(len(unique))
    return start + rank[inverse.reshape(-1)], first[order]


def midpoint_nodes(nodes, pairs) -> tuple[np.ndarray, np.ndarray]:
    """Append one midpoint node per distinct edge of ``pairs`` (M x 2 node ids, in use order),
    numbered in the order of first use; returns the grown node array and each pair's midpoint id
    (the edge-midpoint builder of adtlert/mesh/core.py:27-44)."""

    nodes = np.asarray(nodes, dtype=float)
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    lo, hi = pairs.min(axis=1), pairs.max(axis=1)
    ids, first = first_use_numbers(lo * len(nodes) + hi, len(nodes))
    return np.vstack((nodes, 0.5 * (nodes[lo[first]] + nodes[hi[first]]))), ids


def _orient_ccw(nodes, triangle: list[int]) -> list[int]:
    p0, p1, p2 = (np.asarray(nodes[n], dtype=float) for n in triangle)
    e1, e2 = p1 - p0, p2 - p0
    return triangle if e1[0] * e2[1] - e1[1] * e2[0] > 0.0 else [triangle[0], triangle[2], triangle[1]]


def expand_columnar_triangles(nodes, cells, tol: float = 1e-6):
    """For meshes whose cells each span two adjacent node columns (a node pair in one column,
    one node in the next), add the missing half of every strip quad, creating a bottom node where
    a column is one node short; ``None`` for any other mesh (adtlert/mesh/core.py:466-540)."""

    nodes, cells = np.asarray(nodes, dtype=float), np.asarray(cells, dtype=np.int64)
    if nodes.shape[0] == 0 or cells.shape[0] == 0:
        return None
    columns: list[list[int]] = []
    for node in np.argsort(nodes[:, 0], kind="mergesort").tolist():
        if columns and abs(nodes[node, 0] - nodes[columns[-1][0], 0]) <= tol:
            columns[-1].append(node)
        else:
            columns.append([node])
    sizes = [len(c) for c in columns]
    if len(columns) < 10 or min(sizes) < 2 or max(sizes) - min(sizes) > 1:
        return None
    column_of = np.full(nodes.shape[0], -1, dtype=np.int64)
    row_of = np.full(nodes.shape[0], -1, dtype=np.int64)
    for column_id, column in enumerate(columns):
        column.sort(key=lambda n: (-nodes[n, 1], nodes[n, 0]))
        for row, node in enumerate(column):
            column_of[node], row_of[node] = column_id, row
    expanded_nodes = nodes.tolist()
    expanded, parents = [], []
    for parent, cell in enumerate(cells):
        column_ids, rows = column_of[cell], row_of[cell]
        unique, counts = np.unique(column_ids, return_counts=True)
        if unique.shape[0] != 2 or unique[1] != unique[0] + 1 or sorted(counts.tolist()) != [1, 2]:
            return None
        pair_column, lone_column = int(unique[np.argmax(counts)]), int(unique[np.argmin(counts)])
        pair = column_ids == pair_column
        order = np.argsort(rows[pair])
        pair_nodes, pair_rows = cell[pair][order], rows[pair][order]
        if pair_rows[1] != pair_rows[0] + 1:
            return None
        lone_row = int(rows[~pair][0])
        if lone_row not in pair_rows:
            return None
        missing_row = int(pair_rows[1] if lone_row == pair_rows[0] else pair_rows[0])
        lone = columns[lone_column]
        if missing_row >= len(lone):
            if missing_row != len(lone) or len(lone) + 1 != max(sizes):
                return None
            depth = nodes[int(pair_nodes[1]), 1] - nodes[columns[pair_column][0], 1]
            expanded_nodes.append([float(nodes[lone[0], 0]), float(nodes[lone[0], 1] + depth)])
            lone.append(len(expanded_nodes) - 1)
        missing = int(lone[missing_row])
        if missing in cell.tolist():
            return None
        expanded += [cell.tolist(), _orient_ccw(expanded_nodes, [missing, int(pair_nodes[0]), int(pair_nodes[1])])]
        parents += [parent, parent]
    return np.asarray(expanded_nodes), np.asarray(expanded, dtype=np.int64), np.asarray(parents, dtype=np.int64)


def locate_points(nodes, cells, points, tol: float = 1e-4) -> tuple[np.ndarray, np.ndarray]:
    """Containing cell and interpolation weights of each point; a node within ``tol`` wins and
    takes the first cell using it (adtlert/mesh/core.py:199-324)."""

    cell_ids = np.full(len(points), -1, dtype=np.int64)
    weights = np.zeros((len(points), cells.shape[1]))
    for i, point in enumerate(points):
        distance = np.linalg.norm(nodes - point, axis=1)
        nearest = int(np.argmin(distance))
        if distance[nearest] <= tol:
            hits = np.flatnonzero((cells == nearest).any(axis=1))
            if hits.size:
                cell_ids[i] = hits[0]
                weights[i, int(np.flatnonzero(cells[hits[0]] == nearest)[0])] = 1.0
                continue
        if cells.shape[1] == 3:
            a = nodes[cells[:, 0]]
            m = np.stack((nodes[cells[:, 1]] - a, nodes[cells[:, 2]] - a), axis=-1)
            local = np.linalg.solve(m, (point - a)[..., None])[..., 0]
            bary = np.column_stack((1.0 - local.sum(1), local))
            hits = np.flatnonzero(np.all((bary >= -tol) & (bary <= 1.0 + tol), axis=1))
            if hits.size:
                cell_ids[i], weights[i] = hits[0], bary[hits[0]]
        else:
            for c, cell in enumerate(cells):
                found = _bilinear_weights(nodes[cell], point, tol)
                if found is not None:
                    cell_ids[i], weights[i] = c, found
                    break
    if np.any(cell_ids < 0):
        raise ValueError("some points could not be located in the mesh")
    return cell_ids, weights


def _q1(xi, eta):
    values = 0.25 * np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
    d_xi = 0.25 * np.array([-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)])
    d_eta = 0.25 * np.array([-(1 - xi), -(1 + xi), 1 + xi, 1 - xi])
    return values, np.stack((d_xi, d_eta), axis=1)


def _bilinear_weights(quad, point, tol):
    """Q1 weights of a point on an edge (linear in the edge) or inside (Newton on the map)."""

    for start in range(4):
        stop = (start + 1) % 4
        edge = quad[stop] - quad[start]
        length_sq = float(edge @ edge)
        if length_sq <= tol * tol:
            continue
        t = float((point - quad[start]) @ edge / length_sq)
        if -tol <= t <= 1.0 + tol:
            t = min(max(t, 0.0), 1.0)
            if np.linalg.norm(point - (quad[start] + t * edge)) <= tol:
                w = np.zeros(4)
                w[start], w[stop] = 1.0 - t, t
                return w
    xi = eta = 0.0
    for _ in range(32):
        values, grads = _q1(xi, eta)
        residual = values @ quad - point
        inside = -1 - tol <= xi <= 1 + tol and -1 - tol <= eta <= 1 + tol
        if np.linalg.norm(residual) <= tol and inside:
            break
        try:
            step = np.linalg.solve(grads.T @ quad, residual)
        except np.linalg.LinAlgError:
            return None
        xi, eta = xi - float(step[0]), eta - float(step[1])
        if np.linalg.norm(step) <= 1e-12:
            break
    if not (-1 - tol <= xi <= 1 + tol and -1 - tol <= eta <= 1 + tol):
        return None
    values, _ = _q1(min(max(xi, -1.0), 1.0), min(max(eta, -1.0), 1.0))
    return None if np.any(values < -tol) or np.any(values > 1 + tol) else values


@dataclass(frozen=True)
class Survey:
    """Electrode positions and ABMN rows; ``-1`` is a remote electrode (adtlert/survey/core.py:23-120)."""

    electrode_positions: np.ndarray
    measurements: np.ndarray

    @classmethod
    def from_arrays(cls, electrode_positions, measurements) -> Survey:
        positions = _as_numpy(electrode_positions, float)
        quads = _as_numpy(measurements, np.int64)
        if positions.ndim != 2 or positions.shape[1] not in (2, 3):
            raise ValueError("electrode_positions must have shape (num_electrodes, 2 or 3)")
        if quads.ndim != 2 or quads.shape[1] != 4:
            raise ValueError("measurements must have shape (num_measurements, 4)")
        if np.any(quads < REMOTE_ELECTRODE):
            raise ValueError(f"measurements contain negative electrode indices other than {REMOTE_ELECTRODE} (remote)")
        if quads.size and np.any(quads >= positions.shape[0]):
            raise ValueError("measurements reference electrodes outside the survey")
        remote = quads == REMOTE_ELECTRODE
        if np.any(remote[:, :2].all(axis=1) | remote[:, 2:].all(axis=1)):
            raise ValueError("each current (AB) and potential (MN) pair needs an electrode in the survey")
        distinct = np.where(remote, -1 - np.arange(4), quads)
        if np.any(np.diff(np.sort(distinct, axis=1), axis=1) == 0):
            raise ValueError("each ABMN measurement must use four distinct electrodes")
        return cls(positions, quads)

    @property
    def electrode_count(self) -> int:
        return int(self.electrode_positions.shape[0])

    @property
    def measurement_count(self) -> int:
        return int(self.measurements.shape[0])

    @property
    def dimension(self) -> int:
        return int(self.electrode_positions.shape[1])

    def measurement_slots(self) -> np.ndarray:
        """ABMN with a remote electrode mapped to the zero slot ``electrode_count``."""

        return np.where(self.measurements == REMOTE_ELECTRODE, self.electrode_count, self.measurements)

    def geometric_factors(self) -> np.ndarray:
        """Half-space ``2 pi / (1/AM - 1/AN - 1/BM + 1/BN)``; terms with a remote electrode vanish."""

        return geometric_factors(self.electrode_positions, self.measurements)


def geometric_factors(positions, measurements) -> np.ndarray:
    positions = _as_numpy(positions, float)
    quads = _as_numpy(measurements, np.int64)
    points = positions[np.clip(quads, 0, None)]
    real = quads != REMOTE_ELECTRODE

    def inverse(i, j):
        distance = np.linalg.norm(points[:, i] - points[:, j], axis=-1)
        with np.errstate(divide="ignore"):
            return np.where(real[:, i] & real[:, j], 1.0 / np.where(distance > 0, distance, np.inf), 0.0)

    return 2.0 * math.pi / (inverse(0, 2) - inverse(0, 3) - inverse(1, 2) + inverse(1, 3))
