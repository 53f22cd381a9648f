"""Element spaces of the 2.5D operator: the input mesh (flat surfaces) or the refined auxiliary
meshes of terrain solves (bilinear quadrilateral strips or triangles, P1 or quadratic).

Restates adtlert/forward/discretization.py:128-575 (``build_discretization`` and its helpers) in
float64 NumPy. The result feeds a device plan (``adt_plan_create``); nothing here runs per model.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .fem import (
    boundary_mass,
    boundary_mass_p2,
    p2_triangle_templates,
    quad_templates,
    robin_coefficients,
    serendipity_templates,
    triangle_templates,
)
from .geometry import Mesh, first_use_numbers, midpoint_nodes


@dataclass(frozen=True)
class Discretization:
    """Finite-element space of one family of solves. ``parent_cell_ids`` maps each geometry
    cell to the input-mesh cell whose conductivity it carries; ``boundary_cells`` index geometry
    cells; ``boundary_geometries`` are the Robin coefficients per wavenumber, (W, boundaries)."""

    name: str
    geometry: Mesh
    parent_cell_ids: np.ndarray
    dof_nodes: np.ndarray
    cell_dofs: np.ndarray
    boundary_dofs: np.ndarray
    stiffness: np.ndarray
    mass: np.ndarray
    boundary_mass: np.ndarray
    boundary_geometries: np.ndarray
    electrode_matrix: np.ndarray
    spd: bool

    @property
    def dof_count(self) -> int:
        return int(self.dof_nodes.shape[0])

    @property
    def boundary_cells(self) -> np.ndarray:
        return self.geometry.boundary_edge_cells


def structured_quads(mesh: Mesh) -> Mesh | None:
    """The quadrilateral strip mesh behind a quad mesh or a columnar half-cell triangle mesh,
    else ``None`` (discretization.py:270-311)."""

    if mesh.is_quadrilateral_mesh:
        return mesh
    expanded = mesh.expand_columnar_cells()
    if expanded is None:
        return None
    triangles, parents = expanded
    nodes = triangles.nodes
    pairs: dict[int, list[np.ndarray]] = {}
    for cell, parent in zip(triangles.cells, parents):
        pairs.setdefault(int(parent), []).append(cell)
    quads = []
    for parent in range(mesh.cell_count):
        pair = pairs.get(parent, [])
        node_ids = np.unique(np.concatenate(pair)) if len(pair) == 2 else np.empty(0, dtype=int)
        if node_ids.size != 4:
            return None
        order = np.argsort(nodes[node_ids, 0])
        left, right = node_ids[order[:2]], node_ids[order[2:]]
        if nodes[left, 0].max() > nodes[right, 0].min() + 1e-6:
            return None
        quads.append([
            left[np.argmin(nodes[left, 1])], right[np.argmin(nodes[right, 1])],
            right[np.argmax(nodes[right, 1])], left[np.argmax(nodes[left, 1])],
        ])
    return Mesh.from_arrays(nodes, np.asarray(quads), surface_node_ids=triangles.surface_node_ids)


def refine_quads(mesh: Mesh) -> tuple[Mesh, np.ndarray]:
    """Split every quad into four through its edge midpoints and center (discretization.py:314-341)."""

    nodes = np.asarray(mesh.nodes, dtype=float)
    q, surface, n = mesh.cells, mesh.surface_node_ids, len(mesh.nodes)
    count = len(q)
    # per quad the events of the incremental builder: midpoints of edges b, r, t, l (new on first
    # use), then the center (always new); surface midpoints follow
    edges = q[:, [0, 1, 1, 2, 2, 3, 3, 0]].reshape(count, 4, 2)
    lo, hi = edges.min(axis=2), edges.max(axis=2)
    keys = np.concatenate((np.column_stack((lo * n + hi, -1 - np.arange(count))).reshape(-1),
                           np.minimum(surface[:-1], surface[1:]) * n + np.maximum(surface[:-1], surface[1:])))
    ids, first = first_use_numbers(keys, n)
    mids = 0.5 * (nodes[lo] + nodes[hi])
    centers = 0.25 * (nodes[q[:, 0]] + nodes[q[:, 1]] + nodes[q[:, 2]] + nodes[q[:, 3]])
    sp_lo, sp_hi = np.minimum(surface[:-1], surface[1:]), np.maximum(surface[:-1], surface[1:])
    events = np.concatenate((np.concatenate((mids, centers[:, None]), axis=1).reshape(-1, 2),
                             0.5 * (nodes[sp_lo] + nodes[sp_hi])))
    points = np.vstack((nodes, events[first]))
    cell_ids = ids[:5 * count].reshape(count, 5)
    b, r, t, left, center = cell_ids.T
    bl, br, tr, tl = q.T
    cells = np.stack((np.stack((bl, b, center, left), 1), np.stack((b, br, r, center), 1),
                      np.stack((center, r, tr, t), 1), np.stack((left, center, t, tl), 1)), axis=1).reshape(-1, 4)
    refined_surface = np.empty(max(2 * len(surface) - 1, 0), dtype=np.int64)
    refined_surface[0::2], refined_surface[1::2] = surface, ids[5 * count:]
    refined = Mesh.from_arrays(points, cells, surface_node_ids=refined_surface)
    return refined, np.repeat(np.arange(count, dtype=np.int64), 4)


def serendipity_topology(mesh: Mesh) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Corner + edge-midpoint dofs of 8-node quads and (end, midpoint, end) boundary dofs
    (discretization.py:344-363)."""

    q, boundary = mesh.cells, mesh.boundary_edges
    pairs = np.concatenate((q[:, [0, 1, 1, 2, 2, 3, 3, 0]].reshape(-1, 2), boundary))
    points, ids = midpoint_nodes(mesh.nodes, pairs)
    cells = np.hstack((q, ids[:4 * len(q)].reshape(-1, 4)))
    return points, cells, np.column_stack((boundary[:, 0], ids[4 * len(q):], boundary[:, 1]))


def _points_on_segments(points: np.ndarray, segments: np.ndarray, tol: float) -> np.ndarray:
    start, edge = segments[:, 0], segments[:, 1] - segments[:, 0]
    length_sq = np.sum(edge * edge, axis=1)
    projection = np.sum((points[:, None, :] - start) * edge, axis=2) / np.maximum(length_sq, tol)
    distance = np.linalg.norm(points[:, None, :] - (start + projection[:, :, None] * edge), axis=2)
    return (projection >= -tol) & (projection <= 1.0 + tol) & (distance <= tol) & (length_sq > tol)


def surface_interpolation(mesh: Mesh, boundary_dofs, dof_count: int, points, tol: float = 1e-5) -> np.ndarray:
    """Rows interpolating surface points from the linear (or, with ``boundary_dofs``, quadratic)
    surface-edge dofs (discretization.py:366-454)."""

    surface_ids = mesh.surface_node_ids
    surface = mesh.surface_nodes
    points = np.asarray(points, dtype=float)
    segments = np.stack((surface[:-1], surface[1:]), axis=1)
    hits = _points_on_segments(points, segments, tol)
    midpoints = None if boundary_dofs is None else {tuple(sorted((a, b))): m for a, m, b in np.asarray(boundary_dofs).tolist()}
    matrix = np.zeros((points.shape[0], dof_count))
    for row, point in enumerate(points):
        distances = np.linalg.norm(surface - point, axis=1)
        nearest = int(np.argmin(distances))
        if distances[nearest] <= tol:
            matrix[row, surface_ids[nearest]] = 1.0
            continue
        segment_ids = np.flatnonzero(hits[row])
        if segment_ids.size == 0:
            raise ValueError("surface point could not be matched to an auxiliary surface edge")
        segment = int(segment_ids[0])
        start, stop = segments[segment]
        edge = stop - start
        length_sq = float(edge @ edge)
        if length_sq <= tol:
            raise ValueError("degenerate surface edge in auxiliary quadrilateral mesh")
        t = min(max(float((point - start) @ edge / length_sq), 0.0), 1.0)
        a, b = int(surface_ids[segment]), int(surface_ids[segment + 1])
        if midpoints is None:
            matrix[row, a], matrix[row, b] = 1.0 - t, t
        else:
            matrix[row, a] = 2.0 * (t - 0.5) * (t - 1.0)
            matrix[row, midpoints[tuple(sorted((a, b)))]] = 4.0 * t * (1.0 - t)
            matrix[row, b] = 2.0 * t * (t - 0.5)
    return matrix


def interpolation(mesh: Mesh, cell_dofs: np.ndarray, dof_count: int, points) -> np.ndarray:
    """Rows interpolating points into linear (P1/Q1) or quadratic (P2) dofs by point location
    (discretization.py:457-482)."""

    cell_ids, weights = mesh.locate_points(points)
    if cell_dofs.shape[1] == 6:
        l1, l2, l3 = weights.T
        weights = np.stack((l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1), 4 * l1 * l2, 4 * l2 * l3, 4 * l3 * l1), -1)
    dofs = cell_dofs[cell_ids]
    matrix = np.zeros((dofs.shape[0], dof_count))
    np.add.at(matrix, (np.repeat(np.arange(dofs.shape[0]), dofs.shape[1]), dofs.reshape(-1)), weights.reshape(-1))
    return matrix


def build_discretization(name: str, mesh: Mesh, survey, wavenumbers, *, auxiliary: bool, refine: bool = False,
                         quadratic: bool = False, quadrature_order: int = 2) -> Discretization:
    """The input-mesh discretization (``auxiliary=False``) or a terrain auxiliary one
    (discretization.py:485-575)."""

    strips = structured_quads(mesh) if auxiliary else None
    parents = np.arange(mesh.cell_count)
    positions = np.asarray(survey.electrode_positions, dtype=float)[:, :2]
    if strips is not None:
        geometry = strips
        if refine:
            geometry, parents = refine_quads(geometry)
        if quadratic:
            dof_nodes, cell_dofs, boundary_dofs = serendipity_topology(geometry)
            stiffness, mass = serendipity_templates(geometry.nodes, geometry.cells)
            bmass = boundary_mass_p2(geometry.boundary_edge_lengths)
        else:
            dof_nodes, cell_dofs, boundary_dofs = geometry.nodes, geometry.cells, geometry.boundary_edges
            stiffness, mass = quad_templates(geometry.nodes, geometry.cells)
            bmass = boundary_mass(geometry.boundary_edge_lengths)
        electrode_matrix = surface_interpolation(geometry, boundary_dofs if quadratic else None, len(dof_nodes), positions)
    else:
        geometry = mesh
        if auxiliary and not quadratic and (expanded := geometry.expand_columnar_cells()) is not None:
            geometry, expanded_parents = expanded
            parents = parents[expanded_parents]
        if refine:
            geometry, refined_parents = geometry.refine_uniform()
            parents = parents[refined_parents]
        if quadratic:
            dof_nodes, cell_dofs, boundary_dofs = geometry.build_quadratic_topology()
        else:
            dof_nodes, cell_dofs, boundary_dofs = geometry.nodes, geometry.cells, geometry.boundary_edges
        if geometry.is_triangle_mesh:
            if quadratic:
                stiffness, mass = p2_triangle_templates(dof_nodes, cell_dofs)
                # the quadratic edge mass is laid out for (end, midpoint, end) dofs while P2
                # triangle boundary dofs are (end, end, midpoint); this pairing is the
                # reference's (adtlert/forward/discretization.py:257-267, mesh/core.py:543-555)
                bmass = boundary_mass_p2(geometry.boundary_edge_lengths)
            else:
                stiffness, mass = triangle_templates(geometry.nodes, geometry.cells, quadrature_order)
                bmass = boundary_mass(geometry.boundary_edge_lengths)
        else:
            if quadratic:
                raise ValueError("quadratic topology is currently implemented for triangle meshes only")
            stiffness, mass = quad_templates(geometry.nodes, geometry.cells)
            bmass = boundary_mass(geometry.boundary_edge_lengths)
        electrode_matrix = interpolation(geometry, cell_dofs, len(dof_nodes), positions)
    geometries = robin_coefficients(geometry.boundary_edge_centers, geometry.boundary_edge_normals,
                                    geometry.surface_edge_mask, geometry.surface_reference_level,
                                    positions.mean(axis=0), np.asarray(wavenumbers, dtype=float))
    return Discretization(
        name=name, geometry=geometry, parent_cell_ids=np.asarray(parents, dtype=np.int64),
        dof_nodes=np.asarray(dof_nodes, dtype=float), cell_dofs=np.asarray(cell_dofs, dtype=np.int64),
        boundary_dofs=np.asarray(boundary_dofs, dtype=np.int64), stiffness=stiffness, mass=mass,
        boundary_mass=bmass, boundary_geometries=geometries, electrode_matrix=electrode_matrix,
        spd=not auxiliary,
    )


def exact_node_indices(dof_nodes, points, tol: float = 1e-6) -> np.ndarray:
    """Indices of the dof nodes coinciding with ``points`` (discretization.py:578-600)."""

    dof_nodes, points = np.asarray(dof_nodes, dtype=float), np.asarray(points, dtype=float)
    lookup: dict[tuple[int, ...], int] = {}
    for node_id, node in enumerate(dof_nodes):
        lookup.setdefault(tuple(np.rint(node / tol).astype(np.int64).tolist()), node_id)
    indices = np.empty(points.shape[0], dtype=np.int64)
    for row, point in enumerate(points):
        nearest = lookup.get(tuple(np.rint(point / tol).astype(np.int64).tolist()))
        if nearest is None:
            distances = np.linalg.norm(dof_nodes - point, axis=1)
            nearest = int(np.argmin(distances))
            if distances[nearest] > tol:
                raise ValueError("point does not coincide with a quadrilateral auxiliary node")
        indices[row] = nearest
    return indices
