"""The vectorized refinements and quadratic topologies against an incremental restatement of the
reference's edge-midpoint builder (adtlert/mesh/core.py:27-44, 326-337, 543-555;
adtlert/forward/discretization.py:314-363): same node numbering, coordinates and cells."""

import numpy as np
import pytest

from adtlert_b200 import Mesh
from adtlert_b200.discretization import refine_quads, serendipity_topology
from cases import terrain_quads, terrain_triangles


class _Builder:
    """Incremental node list: each edge's midpoint is appended on its first use."""

    def __init__(self, nodes):
        self.points = [np.asarray(p, dtype=float) for p in np.asarray(nodes, dtype=float)]
        self.index = {}

    def midpoint(self, a, b):
        key = (a, b) if a < b else (b, a)
        if key not in self.index:
            self.index[key] = len(self.points)
            self.points.append(0.5 * (self.points[key[0]] + self.points[key[1]]))
        return self.index[key]


def _triangle_mesh():
    nodes, cells, surface = terrain_triangles(nx=9, nz=4, seed=3)
    return Mesh.from_arrays(nodes, cells, surface_node_ids=surface)


def _quad_mesh():
    nodes, cells, surface = terrain_quads(nx=7, nz=3)
    return Mesh.from_arrays(nodes, cells, surface_node_ids=surface)


def test_uniform_triangle_refinement_matches_the_incremental_builder():
    mesh = _triangle_mesh()
    builder, cells = _Builder(mesh.nodes), []
    for n0, n1, n2 in mesh.cells.tolist():
        m01, m12, m20 = builder.midpoint(n0, n1), builder.midpoint(n1, n2), builder.midpoint(n2, n0)
        cells += [[n0, m01, m20], [n1, m12, m01], [n2, m20, m12], [m01, m12, m20]]
    surface = mesh.surface_node_ids.tolist()
    expected_surface = [surface[0]]
    for a, b in zip(surface[:-1], surface[1:]):
        expected_surface += [builder.midpoint(a, b), b]
    refined, parents = mesh.refine_uniform()
    assert np.array_equal(refined.nodes, np.asarray(builder.points))
    assert np.array_equal(refined.cells, np.asarray(cells))
    assert np.array_equal(refined.surface_node_ids, expected_surface)
    assert np.array_equal(parents, np.repeat(np.arange(mesh.cell_count), 4))


def test_triangle_quadratic_topology_matches_the_incremental_builder():
    mesh = _triangle_mesh()
    builder = _Builder(mesh.nodes)
    cells = [[a, b, c, builder.midpoint(a, b), builder.midpoint(b, c), builder.midpoint(c, a)]
             for a, b, c in mesh.cells.tolist()]
    boundary = [[a, b, builder.midpoint(a, b)] for a, b in mesh.boundary_edges.tolist()]
    points, ours, ours_boundary = mesh.build_quadratic_topology()
    assert np.array_equal(points, np.asarray(builder.points))
    assert np.array_equal(ours, cells) and np.array_equal(ours_boundary, boundary)


def test_quad_refinement_matches_the_incremental_builder():
    mesh = _quad_mesh()
    builder, cells = _Builder(mesh.nodes), []
    for bl, br, tr, tl in mesh.cells.tolist():
        b, r = builder.midpoint(bl, br), builder.midpoint(br, tr)
        t, left = builder.midpoint(tr, tl), builder.midpoint(tl, bl)
        center = len(builder.points)
        p = builder.points
        builder.points.append(0.25 * (p[bl] + p[br] + p[tr] + p[tl]))
        cells += [[bl, b, center, left], [b, br, r, center], [center, r, tr, t], [left, center, t, tl]]
    surface = mesh.surface_node_ids.tolist()
    expected_surface = [surface[0]]
    for a, c in zip(surface[:-1], surface[1:]):
        expected_surface += [builder.midpoint(a, c), c]
    refined, parents = refine_quads(mesh)
    assert np.array_equal(refined.nodes, np.asarray(builder.points))
    assert np.array_equal(refined.cells, np.asarray(cells))
    assert np.array_equal(refined.surface_node_ids, expected_surface)
    assert np.array_equal(parents, np.repeat(np.arange(mesh.cell_count), 4))


def test_serendipity_topology_matches_the_incremental_builder():
    mesh = _quad_mesh()
    builder = _Builder(mesh.nodes)
    cells = [[bl, br, tr, tl, builder.midpoint(bl, br), builder.midpoint(br, tr), builder.midpoint(tr, tl),
              builder.midpoint(tl, bl)] for bl, br, tr, tl in mesh.cells.tolist()]
    boundary = [[a, builder.midpoint(a, b), b] for a, b in mesh.boundary_edges.tolist()]
    points, ours, ours_boundary = serendipity_topology(mesh)
    assert np.array_equal(points, np.asarray(builder.points))
    assert np.array_equal(ours, cells) and np.array_equal(ours_boundary, boundary)


@pytest.mark.parametrize("mesh_of", [_triangle_mesh, _quad_mesh])
def test_refinement_without_a_surface(mesh_of):
    mesh = mesh_of()
    bare = Mesh.from_arrays(mesh.nodes, mesh.cells)
    refined, _ = bare.refine_uniform() if bare.is_triangle_mesh else refine_quads(bare)
    assert refined.cell_count == 4 * mesh.cell_count
