"""Seeded small 2.5D cases shared by the golden-vector generator and the parity tests.

Every case is raw arrays (mesh nodes and cells, electrode positions, ABMN rows, a
conductivity model, a measurement cotangent and a conductivity direction), so the reference,
the oracle and the CUDA path all start from identical inputs.
"""

from __future__ import annotations

import numpy as np


def structured_section(xs, depths, triangles: bool = True):
    """Nodes and cells of a flat-topped section; ``depths`` are positive, increasing from 0.

    Quads are ``[a, b, c, d]`` counter-clockwise from the upper-left node; triangle meshes split
    each quad as ``[a, d, b], [b, d, c]``.
    """

    xs, zs = np.asarray(xs, dtype=float), -np.asarray(depths, dtype=float)
    grid_x, grid_z = np.meshgrid(xs, zs)
    nodes = np.column_stack((grid_x.ravel(), grid_z.ravel()))
    index = np.arange(nodes.shape[0]).reshape(len(zs), len(xs))
    a = index[:-1, :-1].ravel()
    b = index[:-1, 1:].ravel()
    c = index[1:, 1:].ravel()
    d = index[1:, :-1].ravel()
    if triangles:
        cells = np.stack((np.stack((a, d, b), 1), np.stack((b, d, c), 1)), 1).reshape(-1, 3)
    else:
        cells = np.stack((d, c, b, a), 1)
    return nodes, cells


def dipole_dipole(count: int, max_a: int, max_n: int) -> np.ndarray:
    rows = [
        (i, i + a, i + a * (n + 1), i + a * (n + 2))
        for a in range(1, max_a + 1)
        for n in range(1, max_n + 1)
        for i in range(count)
        if i + a * (n + 2) < count
    ]
    return np.asarray(rows, dtype=np.int64)


def _centroids(nodes, cells):
    return nodes[cells].mean(axis=1)


def layered_model(nodes, cells, rng) -> np.ndarray:
    """Conductivity of a three-layer section with one Gaussian anomaly (seeded)."""

    centers = _centroids(nodes, cells)
    depth = -centers[:, 1]
    depth_span = float(depth.max())
    interfaces = np.sort(rng.uniform(0.1, 0.7, 2)) * depth_span
    layer_rho = 10.0 ** rng.uniform(1.0, 3.0, 3)
    rho = np.where(depth < interfaces[0], layer_rho[0], np.where(depth < interfaces[1], layer_rho[1], layer_rho[2]))
    x0 = rng.uniform(centers[:, 0].min(), centers[:, 0].max())
    z0 = -rng.uniform(0.1, 0.5) * depth_span
    radius = rng.uniform(0.1, 0.25) * depth_span
    contrast = 10.0 ** rng.uniform(-1.0, 1.0)
    r2 = (centers[:, 0] - x0) ** 2 + (centers[:, 1] - z0) ** 2
    rho = rho * contrast ** np.exp(-r2 / (2.0 * radius * radius))
    return 1.0 / rho


def terrain_quads(nx: int = 30, nz: int = 12, dx: float = 2.0):
    """Terrain-following quadrilateral strips (the reference's own terrain test geometry): top
    row of nodes first, cells ``[top-left, top-right, bottom-right, bottom-left]``; the surface
    rises with a slope of 0.03 plus a 0.05 sinusoidal ripple per column."""

    x = np.arange(nx + 1) * dx
    slope = 0.03 + 0.05 * np.sin(np.arange(nx))
    z_top = np.concatenate(([0.0], np.cumsum(slope * dx)))
    offsets = np.concatenate(([0.0], -np.cumsum(np.linspace(0.5, 2.0, nz))))
    nodes = np.asarray([[xi, zt + off] for off in offsets for xi, zt in zip(x, z_top)])
    width = nx + 1
    cells = np.asarray([
        [layer * width + c, layer * width + c + 1, (layer + 1) * width + c + 1, (layer + 1) * width + c]
        for layer in range(nz) for c in range(nx)
    ], dtype=np.int64)
    return nodes, cells, np.arange(width)


def terrain_triangles(nx: int = 36, nz: int = 10, dx: float = 1.5, seed: int = 21):
    """Triangles on a jittered terrain-following grid (columns deliberately not aligned, so the
    mesh is not a columnar strip mesh); surface elevation is a sum of three sinusoids."""

    rng = np.random.default_rng(seed)
    x0 = np.arange(nx + 1) * dx
    depths = np.concatenate(([0.0], np.cumsum(np.linspace(0.6, 2.5, nz))))

    def top(x):
        return 1.2 * np.sin(x / 7.0) + 0.6 * np.sin(x / 3.1 + 1.0) + 0.3 * np.sin(x / 1.7 + 2.0)

    nodes = []
    for d in depths:
        jitter = np.zeros(nx + 1)
        jitter[1:-1] = rng.uniform(-0.2, 0.2, nx - 1) * dx
        x = x0 + jitter
        nodes += [[xi, top(xi) - d] for xi in x]
    nodes = np.asarray(nodes)
    width = nx + 1
    cells = []
    for k in range(nz):
        for i in range(nx):
            a, b = k * width + i, k * width + i + 1
            c, d = (k + 1) * width + i + 1, (k + 1) * width + i
            cells += [[a, d, b], [b, d, c]] if (i + k) % 2 == 0 else [[a, d, c], [a, c, b]]
    return nodes, np.asarray(cells, dtype=np.int64), np.arange(width)


CASES = {
    # Flat P1 triangles, dipole-dipole, exercised with every derivative.
    "tri_flat": {"mesh": "tri", "exact_jacobian": True, "parameters": True, "seed": 3},
    # Flat bilinear quadrilaterals (the reference's own test meshes are quad strips).
    "quad_flat": {"mesh": "quad", "exact_jacobian": False, "parameters": False, "seed": 4},
    # Triangles with remote electrodes: pole-dipole (B remote) and dipole-pole (N remote).
    "tri_pole": {"mesh": "tri", "poles": True, "exact_jacobian": False, "parameters": False, "seed": 5},
    # Terrain quadrilateral strips: H2-refined Q1 fields, serendipity-Q2 numerical primary field.
    "quad_terrain": {"mesh": "terrain_quad", "exact_jacobian": True, "parameters": True, "seed": 6},
    # The same geometry with numerical (FEM) geometric factors.
    "quad_terrain_gf": {"mesh": "terrain_quad", "gf_mode": "numerical", "exact_jacobian": False,
                        "parameters": False, "seed": 7},
    # Unstructured-column terrain triangles: H2-refined P1 fields, P2 numerical primary field.
    "tri_terrain": {"mesh": "terrain_tri", "exact_jacobian": False, "parameters": False, "seed": 8},
}


FLAT_CASES = [name for name, spec in CASES.items() if not spec["mesh"].startswith("terrain")]
TERRAIN_CASES = [name for name, spec in CASES.items() if spec["mesh"].startswith("terrain")]


def _terrain_inputs(spec: dict, rng) -> dict:
    if spec["mesh"] == "terrain_quad":
        nodes, cells, surface = terrain_quads()
    else:
        nodes, cells, surface = terrain_triangles()
    electrodes = nodes[surface[2:-2:2]]
    measurements = dipole_dipole(len(electrodes), 2, 4)
    sigma = layered_model(nodes - np.asarray([0.0, nodes[:, 1].max()]), cells, rng)
    return {
        "nodes": nodes,
        "cells": cells,
        "surface_node_ids": surface,
        "electrodes": electrodes,
        "measurements": measurements,
        "sigma": sigma,
        "cotangent": rng.standard_normal(measurements.shape[0]),
        "direction": rng.standard_normal(cells.shape[0]) * sigma * 1e-2,
        "gf_mode": spec.get("gf_mode", "analytic"),
    }


def case_inputs(name: str) -> dict:
    spec = CASES[name]
    rng = np.random.default_rng(spec["seed"])
    if spec["mesh"].startswith("terrain"):
        out = _terrain_inputs(spec, rng)
        if spec.get("parameters"):
            ids = np.full(out["cells"].shape[0], -1, dtype=np.int64)
            half = out["cells"].shape[0] // 2
            ids[:half] = np.arange(half) // 3
            out["parameter_ids"] = ids
        return out
    xs = np.arange(0.0, 45.0 + 1e-9, 1.5)
    depths = np.concatenate(([0.0], np.cumsum(np.concatenate((np.full(4, 0.75), np.geomspace(1.0, 4.0, 5))))))
    nodes, cells = structured_section(xs, depths, triangles=spec["mesh"] == "tri")
    count = 12
    electrodes = np.column_stack((6.0 + 3.0 * np.arange(count), np.zeros(count)))
    measurements = dipole_dipole(count, 2, 4)
    if spec.get("poles"):
        extra = [(i, -1, i + 2, i + 3) for i in range(0, count - 3, 2)]
        extra += [(i, i + 1, i + 3, -1) for i in range(1, count - 3, 3)]
        measurements = np.concatenate((measurements, np.asarray(extra, dtype=np.int64)))
    sigma = layered_model(nodes, cells, rng)
    out = {
        "nodes": nodes,
        "cells": cells.astype(np.int64),
        "electrodes": electrodes,
        "measurements": measurements,
        "sigma": sigma,
        "cotangent": rng.standard_normal(measurements.shape[0]),
        "direction": rng.standard_normal(cells.shape[0]) * sigma * 1e-2,
    }
    if spec.get("parameters"):
        ids = np.full(cells.shape[0], -1, dtype=np.int64)
        half = cells.shape[0] // 2
        ids[:half] = np.arange(half) // 3
        out["parameter_ids"] = ids
    return out


def box_tetrahedra(nx: int = 6, ny: int = 6, nz: int = 4, relief: float = 0.0, size=(12.0, 12.0, 8.0)):
    """Box (default 12 m x 12 m x 8 m) of hexahedra split into six tetrahedra around the main
    diagonal; ``relief`` bends the top surface (z' = z + relief * depth fraction * sin(x / 4))."""

    xs, ys, zs = np.linspace(0, size[0], nx + 1), np.linspace(0, size[1], ny + 1), np.linspace(-size[2], 0, nz + 1)
    gx, gy, gz = np.meshgrid(xs, ys, zs, indexing="ij")
    gz = gz + relief * (gz - gz.min()) / (gz.max() - gz.min()) * np.sin(gx / 4.0)
    nodes = np.column_stack((gx.ravel(), gy.ravel(), gz.ravel()))
    index = np.arange(nodes.shape[0]).reshape(nx + 1, ny + 1, nz + 1)
    corners = np.stack([
        index[:-1, :-1, :-1], index[1:, :-1, :-1], index[1:, 1:, :-1], index[:-1, 1:, :-1],
        index[:-1, :-1, 1:], index[1:, :-1, 1:], index[1:, 1:, 1:], index[:-1, 1:, 1:],
    ], axis=-1).reshape(-1, 8)
    fans = ((1, 2, 6), (2, 3, 6), (3, 7, 6), (7, 4, 6), (4, 5, 6), (5, 1, 6))
    tets = np.stack([corners[:, [0, a, b, c]] for a, b, c in fans], axis=1).reshape(-1, 4)
    return nodes, tets.astype(np.int64)


CASES3D = {
    # flat box, mixed far-field boundary, analytic singularity removal and geometric factors
    "tet_mixed": {"relief": 0.0, "boundary": "mixed", "seed": 11},
    # flat box, homogeneous Dirichlet far field
    "tet_dirichlet": {"relief": 0.0, "boundary": "dirichlet", "seed": 12},
    # bent top surface: point sources and numerical geometric factors
    "tet_relief": {"relief": 1.0, "boundary": "mixed", "seed": 13},
    # the same three set-ups with ten-node P2 tetrahedra (element_order=2)
    "tet_p2_mixed": {"relief": 0.0, "boundary": "mixed", "seed": 14, "order": 2},
    "tet_p2_dirichlet": {"relief": 0.0, "boundary": "dirichlet", "seed": 15, "order": 2},
    "tet_p2_relief": {"relief": 1.0, "boundary": "mixed", "seed": 16, "order": 2},
}


def case3d_inputs(name: str) -> dict:
    spec = CASES3D[name]
    rng = np.random.default_rng(spec["seed"])
    nodes, cells = box_tetrahedra(nx=12, relief=spec["relief"])
    top = nodes[:, 2] >= nodes[:, 2].max() - 1e-9 if spec["relief"] == 0.0 else None
    line = np.flatnonzero(np.isclose(nodes[:, 1], 6.0) & (np.isclose(nodes[:, 2], nodes[:, 2].max()) if top is None else top))
    if spec["relief"] != 0.0:
        # surface nodes of the bent box: the highest node of every (x, y) column on y = 6
        columns = np.flatnonzero(np.isclose(nodes[:, 1], 6.0))
        line = np.asarray([c[np.argmax(nodes[c, 2])] for c in np.split(columns, len(columns) // 5)])
    line = line[np.argsort(nodes[line, 0])]
    electrodes = nodes[line]
    count = len(electrodes)
    rows = [(i, i + 1, i + 1 + n, i + 2 + n) for n in range(1, 4) for i in range(count) if i + 2 + n < count]
    rows += [(i, -1, i + 2, i + 3) for i in range(0, count - 3, 2)]
    measurements = np.asarray(rows, dtype=np.int64)
    centers = nodes[cells].mean(axis=1)
    sigma = np.full(len(cells), 0.01)
    r2 = (centers[:, 0] - 6.0) ** 2 + (centers[:, 1] - 6.0) ** 2 + (centers[:, 2] + 3.0) ** 2
    sigma = sigma * (1.0 + 2.0 * np.exp(-r2 / 8.0)) * np.exp(0.1 * rng.standard_normal(len(cells)))
    return {
        "nodes": nodes,
        "cells": cells,
        "electrodes": electrodes,
        "measurements": measurements,
        "sigma": sigma,
        "cotangent": rng.standard_normal(len(measurements)),
        "direction": rng.standard_normal(len(cells)) * sigma * 1e-2,
        "boundary": spec["boundary"],
        "order": spec.get("order", 1),
    }


def grid_survey_3d():
    """The shape of the 3D benchmark survey at a test-sized mesh: a 12 x 8 surface grid of
    electrodes at 4 m spacing (96) on a 52 m x 36 m x 16 m box of 13.8k tetrahedra, dipole-dipole
    lines in x and y (a <= 3, n <= 6) plus cross-line quadrupoles, every electrode both a current
    and a receiver electrode: 192 field columns with singularity removal."""

    nodes, cells = box_tetrahedra(nx=26, ny=18, nz=6, size=(52.0, 36.0, 16.0))
    grid = np.stack(np.meshgrid(4.0 + 4.0 * np.arange(12), 4.0 + 4.0 * np.arange(8), indexing="ij"), -1)
    electrodes = np.concatenate((grid.reshape(-1, 2), np.zeros((96, 1))), axis=1)
    index = np.arange(96).reshape(12, 8)
    lines = [index[:, j] for j in range(8)] + [index[i, :] for i in range(12)]
    rows = []
    for line in lines:
        count = len(line)
        for a in (1, 2, 3):
            for n in range(1, 7):
                for i in range(count - a * (n + 2)):
                    rows.append((line[i], line[i + a], line[i + a * (n + 1)], line[i + a * (n + 2)]))
    for i in range(11):
        for j in range(7):
            rows.append((index[i, j], index[i, j + 1], index[i + 1, j], index[i + 1, j + 1]))
    measurements = np.asarray(rows, dtype=np.int64)
    rng = np.random.default_rng(21)
    centers = nodes[cells].mean(axis=1)
    sigma = np.full(len(cells), 0.01)
    for cx, cy, cz, r, factor in ((16.0, 12.0, -4.0, 5.0, 10.0), (34.0, 22.0, -6.0, 6.0, 0.1)):
        inside = np.sum((centers - (cx, cy, cz)) ** 2, axis=1) < r * r
        sigma[inside] *= factor
    return {"nodes": nodes, "cells": cells, "electrodes": electrodes, "measurements": measurements,
            "sigma": sigma * np.exp(0.05 * rng.standard_normal(len(cells)))}
