"""Seeded synthetic sections, surveys and models with the shapes of the benchmark workloads.

``flat_section`` builds the 2.5D flat workload: a 120 m x 40 m section of P1 triangles, 1 m
columns, 20 layers of 0.5 m then 20 geometrically graded layers to 40 m depth (121 x 41 =
4961 nodes, 9600 triangles), 48 surface electrodes at 2 m spacing from x = 13 m, and a
dipole-dipole survey with a <= 6, n <= 8 (1232 rows; a <= 6, n <= 3 gives 612).

``terrain_section`` + ``correlated_model`` build the 2.5D terrain workload: a 200 m x 50 m
section of 40,000 P1 triangles under a surface that is a seeded sum of three sinusoids, interior
node columns jittered so the mesh is not a columnar strip mesh, 96 surface electrodes at 1 m,
2538 mixed Wenner-Schlumberger + dipole-dipole rows, and a log-normal resistivity with a 5 m
correlation length.

``box_section`` + ``grid_survey`` + ``ellipsoid_model`` build the 3D workload: a 60 m x 40 m x
20 m box of structured tetrahedra (60 x 40 x 17 hexahedra of six tetrahedra: 244,800 cells,
45,018 nodes), a 12 x 8 surface grid of electrodes at 4 m spacing, 4000 dipole-dipole rows
along the grid's x and y lines, and a 100 ohm-m background with three seeded ellipsoids.
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


def box_section(nx: int = 60, ny: int = 40, nz: int = 17, size=(60.0, 40.0, 20.0)):
    """Box [0, sx] x [0, sy] x [-sz, 0] of nx x ny x nz hexahedra, each split into six
    tetrahedra around its main diagonal: (nodes, cells)."""

    xs, ys, zs = np.linspace(0, size[0], nx + 1), np.linspace(0, size[1], ny + 1), np.linspace(-size[2], 0, nz + 1)
    gx, gy, gz = np.meshgrid(xs, ys, zs, indexing="ij")
    nodes = np.column_stack((gx.ravel(), gy.ravel(), gz.ravel()))
    index = np.arange(nodes.shape[0]).reshape(nx + 1, ny + 1, nz + 1)
    corners = np.stack([
        index[:-1, :-1, :-1], index[1:, :-1, :-1], index[1:, 1:, :-1], index[:-1, 1:, :-1],
        index[:-1, :-1, 1:], index[1:, :-1, 1:], index[1:, 1:, 1:], index[:-1, 1:, 1:],
    ], axis=-1).reshape(-1, 8)
    fans = ((1, 2, 6), (2, 3, 6), (3, 7, 6), (7, 4, 6), (4, 5, 6), (5, 1, 6))
    cells = np.stack([corners[:, [0, a, b, c]] for a, b, c in fans], axis=1).reshape(-1, 4)
    return nodes, cells.astype(np.int64)


def grid_survey(rows: int = 4000, seed: int = 4, shape=(12, 8), spacing: float = 4.0, origin=(8.0, 6.0)):
    """Surface electrodes on a grid and ``rows`` distinct dipole-dipole quadrupoles drawn (seeded)
    from the dipoles of neighbouring electrodes along the grid's x and y lines."""

    gx, gy = np.meshgrid(origin[0] + spacing * np.arange(shape[0]), origin[1] + spacing * np.arange(shape[1]),
                         indexing="ij")
    count = shape[0] * shape[1]
    electrodes = np.column_stack((gx.ravel(), gy.ravel(), np.zeros(count)))
    idx = np.arange(count).reshape(shape)
    dipoles = [(idx[i, j], idx[i + 1, j]) for i in range(shape[0] - 1) for j in range(shape[1])]
    dipoles += [(idx[i, j], idx[i, j + 1]) for i in range(shape[0]) for j in range(shape[1] - 1)]
    if rows > len(dipoles) * (len(dipoles) - 1):
        raise ValueError("more rows than distinct dipole pairs")
    rng = np.random.default_rng(seed)
    quads: set[tuple[int, int, int, int]] = set()
    while len(quads) < rows:
        (a, b), (m, n) = dipoles[rng.integers(len(dipoles))], dipoles[rng.integers(len(dipoles))]
        if len({a, b, m, n}) == 4:
            quads.add((int(a), int(b), int(m), int(n)))
    return electrodes, np.asarray(sorted(quads), dtype=np.int64)


def ellipsoid_model(nodes, cells, seed: int, footprint=((8.0, 52.0), (6.0, 34.0))) -> np.ndarray:
    """Float32 conductivity: 100 ohm-m background with three ellipsoids (semi-axes U(2,8) m,
    centres inside the electrode footprint at depth U(2,12) m, resistivity log-uniform in
    10-1000 ohm-m) at cell centroids."""

    rng = np.random.default_rng(seed)
    centers = nodes[cells].mean(axis=1)
    rho = np.full(len(cells), 100.0)
    for _ in range(3):
        c = np.array([rng.uniform(*footprint[0]), rng.uniform(*footprint[1]), -rng.uniform(2.0, 12.0)])
        axes = rng.uniform(2.0, 8.0, 3)
        inside = np.sum(((centers - c) / axes) ** 2, axis=1) <= 1.0
        rho[inside] = 10.0 ** rng.uniform(1.0, 3.0)
    return (1.0 / rho).astype(np.float32)


def wenner_schlumberger(count: int, max_a: int, max_n: int) -> np.ndarray:
    """ABMN rows A = i, M = i + n a, N = i + (n + 1) a, B = i + (2n + 1) a."""

    rows = [
        (i, i + (2 * n + 1) * a, i + n * a, i + (n + 1) * a)
        for a in range(1, max_a + 1)
        for n in range(1, max_n + 1)
        for i in range(count)
        if i + (2 * n + 1) * a < count
    ]
    return np.asarray(rows, dtype=np.int64).reshape(-1, 4)


def terrain_section(seed: int = 7):
    """The terrain workload: (nodes, cells, surface node ids, electrode positions, ABMN rows).

    x from 0 to 200 m in 1 m columns, 100 layers graded from 0.2 m at the surface to 50 m depth,
    each quad split into two triangles (40,000 cells); the surface is z(x) = sum_i A_i sin(2 pi x
    / L_i + p_i) with A_i ~ U(0, 5/3) m, L_i ~ U(20, 100) m, p_i ~ U(0, 2 pi), every layer
    follows it, and interior nodes move by U(-0.05, 0.05) m in x. Electrodes: the 96 surface
    nodes from x = 52 m; rows: Wenner-Schlumberger a <= 2, n <= 6 and dipole-dipole a <= 3,
    n <= 6 (2538).
    """

    rng = np.random.default_rng(seed)
    xs = np.arange(201, dtype=float)
    steps = np.geomspace(0.2, 1.0, 100)
    depths = np.concatenate(([0.0], np.cumsum(steps * 50.0 / steps.sum())))
    amp, length, phase = rng.uniform(0.0, 5.0 / 3.0, 3), rng.uniform(20.0, 100.0, 3), rng.uniform(0.0, 2 * np.pi, 3)

    def surface(x):
        return sum(a * np.sin(2 * np.pi * x / w + p) for a, w, p in zip(amp, length, phase))

    gx, gd = np.meshgrid(xs, depths)
    gz = surface(gx) - gd
    jitter = rng.uniform(-0.05, 0.05, gx.shape)
    jitter[0, :] = jitter[-1, :] = jitter[:, 0] = jitter[:, -1] = 0.0  # surface, base and sides stay
    nodes = np.column_stack(((gx + jitter).ravel(), gz.ravel()))
    index = np.arange(nodes.shape[0]).reshape(gx.shape)
    ul, ur = index[:-1, :-1].ravel(), index[:-1, 1:].ravel()
    ll, lr = index[1:, :-1].ravel(), index[1:, 1:].ravel()
    cells = np.stack((np.stack((ul, ll, ur), 1), np.stack((ur, ll, lr), 1)), 1).reshape(-1, 3)
    surface_ids = index[0]
    electrodes = nodes[surface_ids[52:148]]
    rows = np.concatenate((wenner_schlumberger(96, 2, 6), dipole_dipole(96, 3, 6)))
    return nodes, cells.astype(np.int64), surface_ids.astype(np.int64), electrodes, rows


def correlated_model(nodes, cells, seed: int, correlation: float = 5.0, spacing: float = 0.5) -> np.ndarray:
    """Float32 conductivity 1 / rho with log10 rho ~ N(2, 0.4^2): white noise on a ``spacing`` grid
    over the mesh's bounding box, Gaussian-filtered in Fourier space to the ``correlation`` length,
    rescaled to unit variance and sampled at the nearest grid point of every cell centroid."""

    rng = np.random.default_rng(seed)
    lo, hi = nodes.min(axis=0), nodes.max(axis=0)
    shape = tuple(int(np.ceil((h - l) / spacing)) + 1 for l, h in zip(lo, hi))
    noise = rng.standard_normal(shape)
    kx = np.fft.fftfreq(shape[0], spacing)[:, None]
    kz = np.fft.fftfreq(shape[1], spacing)[None, :]
    kernel = np.exp(-2.0 * (np.pi * correlation) ** 2 * (kx ** 2 + kz ** 2))
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * kernel))
    field = (field - field.mean()) / field.std()
    centers = nodes[cells].mean(axis=1)
    ij = np.clip(np.rint((centers - lo) / spacing).astype(int), 0, np.array(shape) - 1)
    log_rho = 2.0 + 0.4 * field[ij[:, 0], ij[:, 1]]
    return (1.0 / 10.0 ** log_rho).astype(np.float32)


def infiltration_series(nodes, cells, steps: int = 365, seed: int = 0, max_depth: float = 8.0) -> np.ndarray:
    """(steps, cells) float64 resistivity of the time-lapse workload: the seeded layered model
    with an infiltration front whose depth grows monotonically, f(t) = max_depth (t / (steps -
    1))^0.7, and the resistivity above the front multiplied by one factor c ~ U(0.3, 0.7)."""

    base = 1.0 / layered_model(nodes, cells, seed).astype(float)
    depth = -nodes[cells].mean(axis=1)[:, 1]
    factor = np.random.default_rng(seed + 7919).uniform(0.3, 0.7)
    fronts = max_depth * (np.arange(steps) / max(steps - 1, 1)) ** 0.7
    return np.where(depth[None, :] < fronts[:, None], base[None, :] * factor, base[None, :])
