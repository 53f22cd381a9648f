"""Seeded synthetic sections, surveys and models with the shapes of the benchmark workloads.

``flat_section`` builds the 2.5D flat workload: a 120 m x 40 m section of P1 triangles, 1 m
columns, 20 layers of 0.5 m then 20 geometrically graded layers to 40 m depth (121 x 41 =
4961 nodes, 9600 triangles), 48 surface electrodes at 2 m spacing from x = 13 m, and a
dipole-dipole survey with a <= 6, n <= 8 (1232 rows; a <= 6, n <= 3 gives 612).
"""

from __future__ import annotations

import numpy as np


def structured_section(xs, depths, triangles: bool = True):
    """Nodes and cells of a flat-topped section (``depths`` positive, increasing from 0).

    Quads are counter-clockwise from the lower-left node; triangles split every quad along the
    upper-right / lower-left diagonal.
    """

    xs, zs = np.asarray(xs, dtype=float), -np.asarray(depths, dtype=float)
    grid_x, grid_z = np.meshgrid(xs, zs)
    nodes = np.column_stack((grid_x.ravel(), grid_z.ravel()))
    index = np.arange(nodes.shape[0]).reshape(len(zs), len(xs))
    ul, ur = index[:-1, :-1].ravel(), index[:-1, 1:].ravel()
    lr, ll = index[1:, 1:].ravel(), index[1:, :-1].ravel()
    if triangles:
        cells = np.stack((np.stack((ul, ll, ur), 1), np.stack((ur, ll, lr), 1)), 1).reshape(-1, 3)
    else:
        cells = np.stack((ll, lr, ur, ul), 1)
    return nodes, cells.astype(np.int64)


def dipole_dipole(count: int, max_a: int, max_n: int) -> np.ndarray:
    rows = [
        (i, i + a, i + a * (n + 1), i + a * (n + 2))
        for a in range(1, max_a + 1)
        for n in range(1, max_n + 1)
        for i in range(count)
        if i + a * (n + 2) < count
    ]
    return np.asarray(rows, dtype=np.int64).reshape(-1, 4)


def flat_section(max_n: int = 8):
    """The flat benchmark section: (nodes, cells, electrode positions, ABMN rows)."""

    xs = np.linspace(0.0, 120.0, 121)
    steps = np.concatenate((np.full(20, 0.5), np.geomspace(0.6, 3.7, 20)))
    steps[20:] *= (40.0 - 10.0) / steps[20:].sum()
    depths = np.concatenate(([0.0], np.cumsum(steps)))
    nodes, cells = structured_section(xs, depths)
    electrodes = np.column_stack((13.0 + 2.0 * np.arange(48), np.zeros(48)))
    return nodes, cells, electrodes, dipole_dipole(48, 6, max_n)


def layered_model(nodes, cells, seed: int) -> np.ndarray:
    """Float32 conductivity: three layers (interfaces at U(2,8) m and U(10,25) m depth,
    resistivity log-uniform in 10-1000 ohm-m) times two Gaussian anomalies (radius U(3,8) m,
    contrast 10^U(-1,1), centre x in U(20,100), depth in U(3,25)) at cell centroids."""

    rng = np.random.default_rng(seed)
    centers = nodes[cells].mean(axis=1)
    depth = -centers[:, 1]
    first, second = rng.uniform(2.0, 8.0), rng.uniform(10.0, 25.0)
    rho_layers = 10.0 ** rng.uniform(1.0, 3.0, 3)
    rho = np.where(depth < first, rho_layers[0], np.where(depth < second, rho_layers[1], rho_layers[2]))
    for _ in range(2):
        x0, z0 = rng.uniform(20.0, 100.0), -rng.uniform(3.0, 25.0)
        radius, contrast = rng.uniform(3.0, 8.0), 10.0 ** rng.uniform(-1.0, 1.0)
        r2 = (centers[:, 0] - x0) ** 2 + (centers[:, 1] - z0) ** 2
        rho = rho * contrast ** np.exp(-r2 / (2.0 * radius * radius))
    return (1.0 / rho).astype(np.float32)
