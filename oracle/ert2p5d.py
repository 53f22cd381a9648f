"""FP64 NumPy/SciPy restatement of AD-TLERT's flat 2.5D forward and sensitivity path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the product never imports this.

The algorithm follows the reference step by step; each function names the reference lines it
restates (paths are relative to the AD-TLERT project root). The sparse direct solve uses SciPy's
SuperLU (the reference calls cuDSS through nvmath-python, ``adtlert/forward/cudss.py:24-122``;
a direct solve is exact up to rounding, so the choice of factorization does not change the
result beyond rounding). Everything is evaluated in float64.
"""

from __future__ import annotations

import heapq
import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl
from scipy.special import k0, k1, roots_laguerre, roots_legendre

PYGIMLI_ELECTRODE_RADIUS_FRACTION = 1.0 / 6.0  # adtlert/forward/ert2p5d.py:61


# ---------------------------------------------------------------------------------------------
# wavenumber quadrature: adtlert/forward/integration.py:23-49
# ---------------------------------------------------------------------------------------------
def wavenumber_bounds(electrodes: np.ndarray) -> tuple[float, float]:
    """Half the smallest and twice the largest electrode separation (integration.py:23-29)."""

    distances = np.linalg.norm(electrodes[:, None, :] - electrodes[None, :, :], axis=-1)
    positive = distances[distances > 0.0]
    return float(positive.min() / 2.0), float(positive.max() * 2.0)


def inverse_cosine_weights(r_min: float, r_max: float) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Legendre in sqrt(k) on [0, k0] plus a 4-point Gauss-Laguerre tail (integration.py:32-49)."""

    k_0 = 1.0 / (2.0 * r_min)
    points, weights = roots_legendre(max(int(6.0 * np.log10(r_max / r_min)), 4))
    points, weights = 0.5 * (points + 1.0), 0.5 * weights
    tail_points, tail_weights = roots_laguerre(4)
    wavenumbers = np.concatenate((k_0 * points * points, k_0 * (tail_points + 1.0)))
    quadrature = np.concatenate(
        (2.0 * k_0 * points * weights / np.pi, k_0 * np.exp(tail_points) * tail_weights / np.pi)
    )
    return wavenumbers, quadrature


# ---------------------------------------------------------------------------------------------
# mesh metadata: adtlert/mesh/core.py:73-196, 199-324
# ---------------------------------------------------------------------------------------------
def boundary_topology(cells: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Sorted boundary edges and the first cell owning each (core.py:73-100)."""

    edges = np.sort(np.stack((cells, np.roll(cells, -1, axis=1)), axis=-1), axis=-1)
    unique, first, counts = np.unique(edges.reshape(-1, 2), axis=0, return_index=True, return_counts=True)
    boundary = counts == 1
    return unique[boundary], first[boundary] // cells.shape[1]


def boundary_geometry(nodes, cells, edges, edge_cells):
    """Edge centers, lengths and outward unit normals (core.py:103-121)."""

    edge_nodes = nodes[edges]
    centers = edge_nodes.mean(axis=1)
    vectors = edge_nodes[:, 1] - edge_nodes[:, 0]
    lengths = np.linalg.norm(vectors, axis=1)
    normals = np.stack((vectors[:, 1], -vectors[:, 0]), axis=1) / lengths[:, None]
    outward = np.sum(normals * (centers - nodes[cells[edge_cells]].mean(axis=1)), axis=1) >= 0.0
    return centers, lengths, normals * np.where(outward, 1.0, -1.0)[:, None]


def surface_path(nodes: np.ndarray, edges: np.ndarray, tol: float = 1e-8) -> list[int]:
    """Dijkstra along boundary edges from the upper-left to the upper-right corner (core.py:124-174)."""

    boundary_nodes = np.unique(edges)
    x = nodes[boundary_nodes, 0]

    def corner(extreme):
        candidates = boundary_nodes[np.abs(x - extreme) <= tol].tolist()
        return int(max(candidates, key=lambda node: (nodes[node, 1], -nodes[node, 0])))

    start, stop = corner(float(x.min())), corner(float(x.max()))
    centers_y = nodes[edges].mean(axis=1)[:, 1]
    lengths = np.linalg.norm(nodes[edges[:, 1]] - nodes[edges[:, 0]], axis=1)
    span = max(float(centers_y.max() - centers_y.min()), tol)
    adjacency = {int(node): [] for node in boundary_nodes}
    for (a, b), cy, length in zip(edges.tolist(), centers_y, lengths):
        cost = float(length * (1.0 + 100.0 * (centers_y.max() - cy) / span))
        adjacency[a].append((b, cost))
        adjacency[b].append((a, cost))
    dist, prev, seen, heap = {start: 0.0}, {}, set(), [(0.0, start)]
    while heap:
        d, node = heapq.heappop(heap)
        if node in seen:
            continue
        seen.add(node)
        if node == stop:
            break
        for nb, cost in adjacency[node]:
            if d + cost < dist.get(nb, float("inf")):
                dist[nb], prev[nb] = d + cost, node
                heapq.heappush(heap, (d + cost, nb))
    if start == stop:
        return [start]
    if stop not in prev:
        return [start, stop]
    path = [stop]
    while path[-1] != start:
        path.append(prev[path[-1]])
    return path[::-1]


def locate_points(nodes, cells, points, tol: float = 1e-4):
    """Containing cell and interpolation weights; a node within ``tol`` wins (core.py:199-324)."""

    cell_ids = np.full(len(points), -1)
    weights = np.zeros((len(points), cells.shape[1]))
    for p, point in enumerate(points):
        distances = np.linalg.norm(nodes - point, axis=1)
        nearest = int(np.argmin(distances))
        if distances[nearest] <= tol:
            adjacent = np.flatnonzero(np.any(cells == nearest, axis=1))
            if adjacent.size:
                cell_ids[p] = adjacent[0]
                weights[p, int(np.flatnonzero(cells[adjacent[0]] == nearest)[0])] = 1.0
                continue
        if cells.shape[1] == 3:
            origins = nodes[cells[:, 0]]
            transforms = np.stack((nodes[cells[:, 1]] - origins, nodes[cells[:, 2]] - origins), axis=-1)
            local = np.linalg.solve(transforms, (point - origins)[..., None])[..., 0]
            bary = np.column_stack((1.0 - local.sum(axis=1), local))
            hits = np.flatnonzero(np.all((bary >= -tol) & (bary <= 1.0 + tol), axis=1))
            if hits.size:
                cell_ids[p], weights[p] = hits[0], bary[hits[0]]
        else:
            for c, cell in enumerate(cells):
                found = _quad_weights(nodes[cell], point, tol)
                if found is not None:
                    cell_ids[p], weights[p] = c, found
                    break
    if np.any(cell_ids < 0):
        raise ValueError("some points could not be located in the mesh")
    return cell_ids, weights


def _bilinear(xi, eta):
    values = 0.25 * np.asarray([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)])
    grads = 0.25 * np.stack(
        (np.asarray([-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)]), np.asarray([-(1 - xi), -(1 + xi), 1 + xi, 1 - xi])), axis=1
    )
    return values, grads


def _quad_weights(quad, point, tol):
    """Q1 weights on an edge (linear) or inside (Newton) (core.py:269-306)."""

    for start in range(4):
        stop = (start + 1) % 4
        edge = quad[stop] - quad[start]
        length_sq = float(edge @ edge)
        if length_sq <= tol * tol:
            continue
        t = float((point - quad[start]) @ edge / length_sq)
        if -tol <= t <= 1.0 + tol:
            t = min(max(t, 0.0), 1.0)
            if float(np.linalg.norm(point - (quad[start] + t * edge))) <= tol:
                w = np.zeros(4)
                w[start], w[stop] = 1.0 - t, t
                return w
    xi = eta = 0.0
    for _ in range(32):
        values, grads = _bilinear(xi, eta)
        residual = values @ quad - point
        if float(np.linalg.norm(residual)) <= tol and -1 - tol <= xi <= 1 + tol and -1 - tol <= eta <= 1 + tol:
            break
        try:
            step = np.linalg.solve(grads.T @ quad, residual)
        except np.linalg.LinAlgError:
            return None
        xi, eta = xi - float(step[0]), eta - float(step[1])
        if float(np.linalg.norm(step)) <= 1e-12:
            break
    if not (-1 - tol <= xi <= 1 + tol and -1 - tol <= eta <= 1 + tol):
        return None
    values, _ = _bilinear(min(max(xi, -1.0), 1.0), min(max(eta, -1.0), 1.0))
    return None if np.any(values < -tol) or np.any(values > 1 + tol) else values


# ---------------------------------------------------------------------------------------------
# element templates: adtlert/fem/triangle.py:94-235, adtlert/forward/discretization.py:223-267,
# adtlert/fem/boundary.py:31-82
# ---------------------------------------------------------------------------------------------
_P1_RULES = {
    1: ([[1 / 3, 1 / 3]], [0.5]),
    2: ([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]], [1 / 6] * 3),
}


def triangle_templates(nodes, cells, quadrature_order: int = 2):
    """P1 stiffness ``|T| G G^T`` and quadrature mass (triangle.py:94-133, 203-235)."""

    points, weights = (np.asarray(v, dtype=float) for v in _P1_RULES[quadrature_order])
    shape = np.stack((1.0 - points[:, 0] - points[:, 1], points[:, 0], points[:, 1]), axis=-1)
    reference = np.asarray([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]])
    cn = nodes[cells]
    jac = np.stack((cn[:, 1] - cn[:, 0], cn[:, 2] - cn[:, 0]), axis=-1)
    grads = np.einsum("eij,nj->eni", np.linalg.inv(jac).transpose(0, 2, 1), reference)
    areas = 0.5 * np.abs(np.linalg.det(jac))
    w = 2.0 * areas[:, None] * weights[None, :]
    stiffness = np.einsum("eid,ejd,eq->eij", grads, grads, w)
    mass = np.einsum("qi,qj,eq->eij", shape, shape, w)
    return stiffness, mass


def quad_templates(nodes, cells):
    """Bilinear Q1 stiffness and mass by 2x2 Gauss (discretization.py:223-267, linear branch)."""

    g = 1.0 / np.sqrt(3.0)
    points = np.asarray([[-g, -g], [g, -g], [g, g], [-g, g]])
    values = np.stack([_bilinear(*p)[0] for p in points])
    grads = np.stack([_bilinear(*p)[1] for p in points])  # (q, i, a)
    cn = nodes[cells]
    jac = np.einsum("cid,qia->cqda", cn, grads)
    physical = np.einsum("qia,cqab->cqib", grads, np.linalg.inv(jac))
    wdet = np.abs(np.linalg.det(jac))
    stiffness = np.einsum("cqid,cqjd,cq->cij", physical, physical, wdet)
    mass = np.einsum("qi,qj,cq->cij", values, values, wdet)
    return stiffness, mass


def robin_coefficients(centers, normals, surface_mask, surface_level, source, k):
    """``k [(r1.n/r1) K1(k r1) + (r2.n/r2) K1(k r2)] / [K0(k r1) + K0(k r2)]`` (boundary.py:43-82)."""

    image = np.asarray([source[0], 2.0 * surface_level - source[1]])
    r1, r2 = centers - source, centers - image
    a1, a2 = np.linalg.norm(r1, axis=1), np.linalg.norm(r2, axis=1)
    out = np.zeros(len(centers))
    valid = np.flatnonzero((a1 > 1e-12) & (a2 > 1e-12) & ~surface_mask)
    den = k0(a1[valid] * k) + k0(a2[valid] * k)
    stable = valid[den > 1e-12]
    num = np.sum(r1[stable] * normals[stable], 1) / a1[stable] * k1(a1[stable] * k) + np.sum(
        r2[stable] * normals[stable], 1
    ) / a2[stable] * k1(a2[stable] * k)
    out[stable] = k * num / den[den > 1e-12]
    return out


def halfspace_primary(nodes, source, k, surface):
    """Unit-resistivity half-space primary field, image source when buried (ert2p5d.py:78-94)."""

    distance = np.linalg.norm(nodes - source, axis=1)
    values = np.zeros(len(nodes))
    if abs(source[1] - surface) <= 1e-8:
        valid = distance > 1e-12
        values[valid] = k0(distance[valid] * k) / np.pi
        return values
    mirrored = np.linalg.norm(nodes - (source[0], 2.0 * surface - source[1]), axis=1)
    valid = (distance > 1e-12) & (mirrored > 1e-12)
    values[valid] = (k0(distance[valid] * k) + k0(mirrored[valid] * k)) / (2.0 * np.pi)
    return values


# ---------------------------------------------------------------------------------------------
# the operator
# ---------------------------------------------------------------------------------------------
class Oracle2p5D:
    """Flat-surface 2.5D operator on the input mesh (``build_discretization("native")``).

    Mirrors ``ERTForward2p5D`` (adtlert/forward/ert2p5d.py:108-1121) for flat triangle (P1) and
    quadrilateral (Q1) meshes.
    """

    def __init__(self, nodes, cells, electrodes, measurements, quadrature_order: int = 2):
        self.nodes = np.asarray(nodes, dtype=float)
        self.cells = np.asarray(cells, dtype=np.int64)
        self.electrodes = np.asarray(electrodes, dtype=float)
        self.measurements = np.asarray(measurements, dtype=np.int64)
        E, C = len(self.electrodes), len(self.cells)
        self.E, self.C, self.N = E, C, len(self.nodes)
        self.K = self.cells.shape[1]
        # quadrature (ert2p5d.py:158)
        self.wavenumbers, self.weights = inverse_cosine_weights(*wavenumber_bounds(self.electrodes))
        self.W = len(self.wavenumbers)
        # boundary + surface metadata (core.py:576-630)
        self.edges, self.edge_cells = boundary_topology(self.cells)
        self.centers, self.lengths, self.normals = boundary_geometry(self.nodes, self.cells, self.edges, self.edge_cells)
        path = np.asarray(surface_path(self.nodes, self.edges))
        pairs = {tuple(sorted(p)) for p in zip(path[:-1].tolist(), path[1:].tolist())}
        self.surface_mask = np.asarray([tuple(e) in pairs for e in self.edges.tolist()], dtype=bool)
        self.surface_level = float(self.nodes[path, 1].mean())
        # templates (discretization.py:540-548)
        if self.K == 3:
            self.stiffness, self.mass = triangle_templates(self.nodes, self.cells, quadrature_order)
        else:
            self.stiffness, self.mass = quad_templates(self.nodes, self.cells)
        self.boundary_mass = self.lengths[:, None, None] * np.asarray([[2.0, 1.0], [1.0, 2.0]]) / 6.0
        center = self.electrodes.mean(axis=0)
        self.robin = np.stack(
            [robin_coefficients(self.centers, self.normals, self.surface_mask, self.surface_level, center, k) for k in self.wavenumbers]
        )  # (W, Nb), discretization.py:549-557
        # electrode interpolation rows (discretization.py:457-482)
        ids, w = locate_points(self.nodes, self.cells, self.electrodes)
        self.electrode_matrix = np.zeros((E, self.N))
        np.add.at(self.electrode_matrix, (np.repeat(np.arange(E), self.K), self.cells[ids].reshape(-1)), w.reshape(-1))
        # sparse pattern (discretization.py:100-125)
        K = self.K
        vol = np.stack((np.repeat(self.cells, K, axis=1).reshape(-1), np.tile(self.cells, (1, K)).reshape(-1)), 1)
        bnd = np.stack((np.repeat(self.edges, 2, axis=1).reshape(-1), np.tile(self.edges, (1, 2)).reshape(-1)), 1)
        unique, inverse = np.unique(np.concatenate((vol, bnd)), axis=0, return_inverse=True)
        inverse = inverse.reshape(-1)
        self.rows, self.cols = unique[:, 0], unique[:, 1]
        self.nnz = len(unique)
        self.volume_slot = inverse[: len(vol)].reshape(C, K * K)
        self.boundary_slot = inverse[len(vol):].reshape(-1, 4)
        # sources (ert2p5d.py:192-208)
        distances = np.linalg.norm(self.nodes[None] - self.electrodes[:, None], axis=2)
        nearest = np.argmin(distances, axis=1)
        self.source_nodes = np.where(distances[np.arange(E), nearest] <= 1e-2, nearest, -1)
        self.source_cells = ids
        # measurement slots with the remote electrode at index E (survey/core.py:77-85)
        q = self.measurements
        self.slots = np.where(q == -1, E, q)
        self._primary = None
        self._refrhs = None
        self._fields_cache = {}

    # -- assembly (ert2p5d.py:252-314) ------------------------------------------------------
    def assemble(self, sigma, robin: bool = True) -> np.ndarray:
        values = np.zeros((self.W, self.nnz))
        k2 = self.wavenumbers**2
        volume = sigma[:, None, None] * (self.stiffness[None] + k2[:, None, None, None] * self.mass[None])
        for w in range(self.W):
            np.add.at(values[w], self.volume_slot.reshape(-1), volume[w].reshape(-1))
            if robin:
                bt = (sigma[self.edge_cells] * self.robin[w])[:, None, None] * self.boundary_mass
                np.add.at(values[w], self.boundary_slot.reshape(-1), bt.reshape(-1))
        return values

    def matrix(self, values_w) -> sp.csr_matrix:
        return sp.csr_matrix((values_w, (self.rows, self.cols)), shape=(self.N, self.N))

    # -- primary field (ert2p5d.py:438-511) -----------------------------------------------------
    def primary(self) -> np.ndarray:
        if self._primary is None:
            surface = float(self.nodes[:, 1].max())
            radii = {}
            for node in set(self.source_nodes.tolist()) - {-1}:
                nb = np.setdiff1d(np.unique(self.cells[np.any(self.cells == node, axis=1)]), [node])
                radii[node] = np.min(np.linalg.norm(self.nodes[nb] - self.nodes[node], axis=1)) if nb.size else None
            out = np.zeros((self.W, self.E, self.N))
            for w, k in enumerate(self.wavenumbers):
                for s, (source, node) in enumerate(zip(self.electrodes, self.source_nodes)):
                    out[w, s] = halfspace_primary(self.nodes, source, k, surface)
                    if node >= 0:
                        r = radii[node]
                        out[w, s, node] = 0.0 if r is None else k0(r * PYGIMLI_ELECTRODE_RADIUS_FRACTION * k) / np.pi
            self._primary = out
        return self._primary

    def reference_rhs(self) -> np.ndarray:
        if self._refrhs is None:
            values = self.assemble(np.ones(self.C))
            up = self.primary()
            self._refrhs = np.stack([(self.matrix(values[w]) @ up[w].T).T for w in range(self.W)])
        return self._refrhs

    def source_resistivities(self, sigma) -> np.ndarray:
        out = np.empty(self.E)
        for e, node in enumerate(self.source_nodes):
            if node >= 0:
                mask = np.any(self.cells == node, axis=1)
                out[e] = np.exp(np.sum(-np.log(sigma[mask])) / np.count_nonzero(mask))
            else:
                out[e] = 1.0 / sigma[self.source_cells[e]]
        return out

    # -- fields (ert2p5d.py:532-553) ------------------------------------------------------------
    def fields(self, sigma):
        key = np.asarray(sigma, dtype=float).tobytes()
        if key in self._fields_cache:
            return self._fields_cache[key]
        sigma = np.asarray(sigma, dtype=float)
        values = self.assemble(sigma)
        primary = self.primary() * self.source_resistivities(sigma)[None, :, None]
        total = np.empty((self.W, self.E, self.N))
        factors = []
        for w in range(self.W):
            A = self.matrix(values[w]).tocsc()
            lu = spl.splu(A)
            factors.append(lu)
            rhs = self.reference_rhs()[w] - (A @ primary[w].T).T
            total[w] = lu.solve(rhs.T).T + primary[w]
        result = (values, total, factors)
        self._fields_cache = {key: result}
        return result

    def integrate(self, fields) -> np.ndarray:
        return np.tensordot(self.weights, fields, axes=([0], [0]))  # ert2p5d.py:560-563

    def normal_reciprocal(self, integrated):
        """(ert2p5d.py:574-589) with the zero remote slot (survey/core.py:16-20)."""

        p = np.pad(integrated @ self.electrode_matrix.T, ((0, 1), (0, 1)))
        a, b, m, n = self.slots.T

        def transfer(src, snk, pos, neg):
            return (p[src, pos] - p[src, neg]) - (p[snk, pos] - p[snk, neg])

        return transfer(a, b, m, n), transfer(m, n, a, b)

    def geometric_factors(self) -> np.ndarray:
        """Analytic ``2 pi / (1/AM - 1/AN - 1/BM + 1/BN)``, remote terms dropped (survey/core.py:87-110)."""

        q = self.measurements
        pts = self.electrodes[np.clip(q, 0, None)]
        real = q != -1

        def inv(p, r):
            d = np.linalg.norm(pts[:, p] - pts[:, r], axis=-1)
            return np.where(real[:, p] & real[:, r], 1.0 / np.where(d > 0, d, 1.0), 0.0)

        return 2.0 * math.pi / (inv(0, 2) - inv(0, 3) - inv(1, 2) + inv(1, 3))

    def resistance(self, sigma) -> np.ndarray:
        _, total, _ = self.fields(sigma)
        n, r = self.normal_reciprocal(self.integrate(total))
        return np.sign(n) * np.sqrt(np.abs(n * r))  # ert2p5d.py:641-645

    def apparent_resistivity(self, sigma, currents=1.0) -> np.ndarray:
        return self.geometric_factors() * self.resistance(sigma) / currents  # ert2p5d.py:709-713

    # -- sensitivities ----------------------------------------------------------------------
    def normal_jacobian(self, sigma, parameter_ids=None, parameter_count=None) -> np.ndarray:
        """``-sum_w w_w (u_M - u_N)^T (K + k^2 M) (u_A - u_B)`` per (row, cell) (ert2p5d.py:984-1010)."""

        _, total, _ = self.fields(sigma)
        phi = np.concatenate((total, np.zeros((self.W, 1, self.N))), axis=1)
        a, b, m, n = self.slots.T
        J = np.zeros((len(a), self.C))
        for w in range(self.W):
            T = self.weights[w] * (self.stiffness + self.wavenumbers[w] ** 2 * self.mass)
            cur = (phi[w, a] - phi[w, b])[:, self.cells]  # (D, C, K)
            rec = (phi[w, m] - phi[w, n])[:, self.cells]
            J -= np.einsum("dci,cij,dcj->dc", rec, T, cur)
        return self._aggregate(J, parameter_ids, parameter_count)

    def _aggregate(self, values, parameter_ids, parameter_count):
        """Sum cell columns into parameters; ``-1`` drops a cell (kernels.py:88-113)."""

        if parameter_ids is None:
            return values
        ids = np.asarray(parameter_ids)
        count = int(ids.max()) + 1 if parameter_count is None else int(parameter_count)
        out = np.zeros(values.shape[:-1] + (count,))
        for p in range(count):
            out[..., p] = values[..., ids == p].sum(axis=-1)
        return out

    def _pair_cotangent(self, normal, reciprocal=None) -> np.ndarray:
        """Scatter of resistance cotangents onto (E, E) electrode potentials (ert2p5d.py:591-629)."""

        E = self.E
        p = np.zeros((E + 1, E + 1))
        a, b, m, n = self.slots.T
        for g, (src, snk, pos, neg) in ((normal, (a, b, m, n)), (reciprocal, (m, n, a, b))):
            if g is None:
                continue
            np.add.at(p, (src, pos), g)
            np.add.at(p, (src, neg), -g)
            np.add.at(p, (snk, pos), -g)
            np.add.at(p, (snk, neg), g)
        return p[:E, :E]

    def cell_gradient(self, phi, lam, robin: bool = True) -> np.ndarray:
        """``-sum_{w,s} lam_ws^T dA_w/dsigma_c phi_ws`` (ert2p5d.py:765-825)."""

        g = np.zeros(self.C)
        for w in range(self.W):
            T = self.stiffness + self.wavenumbers[w] ** 2 * self.mass
            g -= np.einsum("sci,cij,scj->c", lam[w][:, self.cells], T, phi[w][:, self.cells])
            if robin:
                bt = self.robin[w][:, None, None] * self.boundary_mass
                gb = -np.einsum("sbi,bij,sbj->b", lam[w][:, self.edges], bt, phi[w][:, self.edges])
                np.add.at(g, self.edge_cells, gb)
        return g

    def _scale(self, normal, reciprocal):
        return np.sign(reciprocal), np.maximum(np.sqrt(np.abs(normal * reciprocal)), 1e-30)  # ert2p5d.py:647-655

    def vjp(self, sigma, cotangent) -> np.ndarray:
        """Exact VJP of the reciprocity-averaged resistance (ert2p5d.py:835-871)."""

        _, total, factors = self.fields(sigma)
        normal, reciprocal = self.normal_reciprocal(self.integrate(total))
        sign, scale = self._scale(normal, reciprocal)
        common = 0.5 * np.asarray(cotangent) * sign / scale
        pairs = self._pair_cotangent(common * reciprocal, common * normal)
        rhs = pairs @ self.electrode_matrix  # (E, N); ert2p5d.py:631-639
        lam = np.stack([self.weights[w] * factors[w].solve(rhs.T).T for w in range(self.W)])
        return self.cell_gradient(total, lam)

    def exact_jacobian(self, sigma) -> np.ndarray:
        """Exact-derivative rows (ert2p5d.py:1012-1050): the VJP of every unit cotangent."""

        eye = np.eye(len(self.measurements))
        return np.stack([self.vjp(sigma, row) for row in eye])

    def jvp(self, sigma, direction) -> np.ndarray:
        """Tangent solve with the forward factorization (ert2p5d.py:873-890)."""

        _, total, factors = self.fields(sigma)
        normal, reciprocal = self.normal_reciprocal(self.integrate(total))
        dvalues = self.assemble(np.asarray(direction, dtype=float))
        delta = np.stack(
            [factors[w].solve(-(self.matrix(dvalues[w]) @ total[w].T)).T for w in range(self.W)]
        )
        dn, dr = self.normal_reciprocal(self.integrate(delta))
        sign, scale = self._scale(normal, reciprocal)
        return 0.5 * sign * (dn * reciprocal + normal * dr) / scale

    def normal_vjp(self, sigma, cotangent, parameter_ids=None, parameter_count=None) -> np.ndarray:
        """(ert2p5d.py:892-912): no solve, Robin term omitted."""

        _, total, _ = self.fields(sigma)
        pairs = self._pair_cotangent(np.asarray(cotangent, dtype=float)).T
        current = np.einsum("ef,wfn->wen", pairs, total)
        receiver = self.weights[:, None, None] * total
        g = self.cell_gradient(current, receiver, robin=False)
        return self._aggregate(g, parameter_ids, parameter_count)

    def normal_jvp(self, sigma, direction) -> np.ndarray:
        """Gram of ``phi`` against ``-A(delta) phi`` gathered at ABMN (ert2p5d.py:914-943)."""

        _, total, _ = self.fields(sigma)
        dvalues = self.assemble(np.asarray(direction, dtype=float), robin=False)
        gram = np.zeros((self.E, self.E))
        for w in range(self.W):
            gram += self.weights[w] * total[w] @ (-(self.matrix(dvalues[w]) @ total[w].T))
        gram = np.pad(gram, ((0, 1), (0, 1)))
        a, b, m, n = self.slots.T
        return gram[m, a] - gram[m, b] - gram[n, a] + gram[n, b]
