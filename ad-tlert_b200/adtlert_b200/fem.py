"""Host-side set-up of the 2.5D discretizations: quadrature, P1/Q1/P2/serendipity element
templates, boundary terms.

All of this runs once per operator (float64 NumPy/SciPy); the per-model work is on the GPU.
Formulas follow the reference's element math (cited per function).
"""

from __future__ import annotations

import numpy as np
from scipy.special import k0, k1, roots_laguerre, roots_legendre

ELECTRODE_RADIUS_FRACTION = 1.0 / 6.0
"""The primary field at an electrode's own node is K0 at this fraction of the distance to the
nearest neighbouring node (adtlert/forward/ert2p5d.py:61-63)."""


def wavenumber_bounds(positions: np.ndarray) -> tuple[float, float]:
    """Half the smallest and twice the largest electrode separation (adtlert/forward/integration.py:23-29)."""

    diff = positions[:, None, :] - positions[None, :, :]
    distance = np.sqrt(np.sum(diff * diff, axis=-1))
    positive = distance[distance > 0.0]
    return float(positive.min() / 2.0), float(positive.max() * 2.0)


def inverse_cosine_weights(r_min: float, r_max: float) -> tuple[np.ndarray, np.ndarray]:
    """Wavenumbers and weights of the inverse cosine transform: Gauss-Legendre in sqrt(k) on
    [0, 1/(2 r_min)] with max(floor(6 log10(r_max/r_min)), 4) nodes, plus a 4-node Gauss-Laguerre
    tail (adtlert/forward/integration.py:32-49)."""

    k_edge = 0.5 / r_min
    x, w = roots_legendre(max(int(6.0 * np.log10(r_max / r_min)), 4))
    s, ws = 0.5 * (x + 1.0), 0.5 * w
    tx, tw = roots_laguerre(4)
    wavenumbers = np.concatenate((k_edge * s * s, k_edge * (tx + 1.0)))
    weights = np.concatenate((2.0 * k_edge * s * ws / np.pi, k_edge * np.exp(tx) * tw / np.pi))
    return wavenumbers, weights


_TRIANGLE_RULES = {
    1: (np.array([[1 / 3, 1 / 3]]), np.array([0.5])),
    2: (np.array([[1 / 6, 1 / 6], [2 / 3, 1 / 6], [1 / 6, 2 / 3]]), np.full(3, 1 / 6)),
}


def triangle_templates(nodes: np.ndarray, cells: np.ndarray, quadrature_order: int = 2):
    """Unit P1 stiffness |T| G G^T and quadrature mass 2|T| sum_q w_q phi_i phi_j
    (adtlert/fem/triangle.py:94-133, 203-235)."""

    if quadrature_order not in _TRIANGLE_RULES:
        raise ValueError(f"unsupported triangle quadrature order: {quadrature_order}")
    points, weights = _TRIANGLE_RULES[quadrature_order]
    phi = np.column_stack((1.0 - points.sum(1), points))
    p = nodes[cells]
    e1, e2 = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]
    det = e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]
    area = 0.5 * np.abs(det)
    # gradients of the barycentric functions: rows of inv([e1 e2])^T applied to the reference ones
    inv = np.stack((np.stack((e2[:, 1], -e2[:, 0]), 1), np.stack((-e1[:, 1], e1[:, 0]), 1)), 1) / det[:, None, None]
    reference = np.array([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]])
    grads = np.einsum("cij,ni->cnj", inv, reference)
    stiffness = area[:, None, None] * np.einsum("cid,cjd->cij", grads, grads)
    mass = 2.0 * area[:, None, None] * np.einsum("q,qi,qj->ij", weights, phi, phi)[None]
    return stiffness, mass


def quad_templates(nodes: np.ndarray, cells: np.ndarray):
    """Unit bilinear (Q1) stiffness and mass with the 2x2 Gauss rule
    (adtlert/forward/discretization.py:223-267, linear branch)."""

    g = 1.0 / np.sqrt(3.0)
    pts = np.array([[-g, -g], [g, -g], [g, g], [-g, g]])
    xi, eta = pts[:, 0], pts[:, 1]
    values = 0.25 * np.stack(((1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)), -1)
    d_xi = 0.25 * np.stack((-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)), -1)
    d_eta = 0.25 * np.stack((-(1 - xi), -(1 + xi), 1 + xi, 1 - xi), -1)
    ref = np.stack((d_xi, d_eta), -1)  # (q, i, a)
    p = nodes[cells]  # (c, i, d)
    jac = np.einsum("cid,qia->cqda", p, ref)
    inv = np.linalg.inv(jac)
    grads = np.einsum("qia,cqab->cqib", ref, inv)
    wdet = np.abs(np.linalg.det(jac))
    stiffness = np.einsum("cqid,cqjd,cq->cij", grads, grads, wdet)
    mass = np.einsum("qi,qj,cq->cij", values, values, wdet)
    return stiffness, mass


# Six-point degree-4 rule on the reference triangle (Dunavant's published rule; weights sum to
# the reference area 1/2), as adtlert/fem/triangle.py:21-31 tabulates it.
_DEGREE4_POINTS = np.array([
    [0.445948490915965, 0.445948490915965], [0.445948490915965, 0.108103018168070],
    [0.108103018168070, 0.445948490915965], [0.091576213509771, 0.091576213509771],
    [0.091576213509771, 0.816847572980459], [0.816847572980459, 0.091576213509771],
])
_DEGREE4_WEIGHTS = np.array([0.1116907948390055] * 3 + [0.0549758718276610] * 3)


def p2_triangle_templates(nodes: np.ndarray, cells: np.ndarray):
    """Unit P2 stiffness and mass of 6-node triangles (vertices, then midpoints 01, 12, 20) with
    the degree-4 rule (adtlert/fem/triangle.py:140-255)."""

    pts, wts = _DEGREE4_POINTS, _DEGREE4_WEIGHTS
    l2, l3 = pts[:, 0], pts[:, 1]
    l1 = 1.0 - l2 - l3
    values = np.stack((l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1), 4 * l1 * l2, 4 * l2 * l3, 4 * l3 * l1), -1)
    g1, g2, g3 = np.array([-1.0, -1.0]), np.array([1.0, 0.0]), np.array([0.0, 1.0])
    L1, L2, L3 = (x[:, None] for x in (l1, l2, l3))
    reference = np.stack((
        (4 * L1 - 1) * g1, (4 * L2 - 1) * g2, (4 * L3 - 1) * g3,
        4 * (L1 * g2 + L2 * g1), 4 * (L2 * g3 + L3 * g2), 4 * (L3 * g1 + L1 * g3),
    ), axis=-2)  # (q, 6, 2)
    p = nodes[cells[:, :3]]
    jac = np.stack((p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=-1)
    area = 0.5 * np.abs(np.linalg.det(jac))
    grads = np.einsum("eij,qnj->eqni", np.linalg.inv(jac).transpose(0, 2, 1), reference)
    weights = 2.0 * area[:, None] * wts[None, :]
    stiffness = np.einsum("eqid,eqjd,eq->eij", grads, grads, weights)
    mass = np.einsum("qi,qj,eq->eij", values, values, weights)
    return stiffness, mass


def _serendipity(points: np.ndarray):
    xi, eta = points[:, 0], points[:, 1]
    values = np.stack((
        -0.25 * (1 - xi) * (1 - eta) * (1 + xi + eta), -0.25 * (1 + xi) * (1 - eta) * (1 - xi + eta),
        -0.25 * (1 + xi) * (1 + eta) * (1 - xi - eta), -0.25 * (1 - xi) * (1 + eta) * (1 + xi - eta),
        0.5 * (1 - xi * xi) * (1 - eta), 0.5 * (1 + xi) * (1 - eta * eta),
        0.5 * (1 - xi * xi) * (1 + eta), 0.5 * (1 - xi) * (1 - eta * eta),
    ), axis=-1)
    d_xi = np.stack((
        0.25 * (1 - eta) * (2 * xi + eta), 0.25 * (1 - eta) * (2 * xi - eta),
        0.25 * (1 + eta) * (2 * xi + eta), 0.25 * (1 + eta) * (2 * xi - eta),
        -xi * (1 - eta), 0.5 * (1 - eta * eta), -xi * (1 + eta), -0.5 * (1 - eta * eta),
    ), axis=-1)
    d_eta = np.stack((
        0.25 * (1 - xi) * (xi + 2 * eta), 0.25 * (1 + xi) * (-xi + 2 * eta),
        0.25 * (1 + xi) * (xi + 2 * eta), 0.25 * (1 - xi) * (-xi + 2 * eta),
        -0.5 * (1 - xi * xi), -(1 + xi) * eta, 0.5 * (1 - xi * xi), -(1 - xi) * eta,
    ), axis=-1)
    return values, np.stack((d_xi, d_eta), axis=-1)


def serendipity_templates(nodes: np.ndarray, quads: np.ndarray):
    """Unit 8-node serendipity stiffness and mass on bilinear quadrilateral geometry, 3x3 Gauss
    rule (adtlert/forward/discretization.py:159-267, quadratic branch); ``quads`` are the 4
    geometry corners."""

    g, gw = np.polynomial.legendre.leggauss(3)
    pts = np.asarray([[x, y] for y in g for x in g])
    wts = np.asarray([wx * wy for wy in gw for wx in gw])
    xi, eta = pts[:, 0], pts[:, 1]
    geometry = 0.25 * np.stack(
        (np.stack((-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)), -1), np.stack((-(1 - xi), -(1 + xi), 1 + xi, 1 - xi), -1)),
        axis=-1,
    )  # (q, 4, 2)
    values, reference = _serendipity(pts)
    jac = np.einsum("cid,qia->cqda", nodes[quads], geometry)
    grads = np.einsum("qia,cqab->cqib", reference, np.linalg.inv(jac))
    wdet = np.abs(np.linalg.det(jac)) * wts
    stiffness = np.einsum("cqid,cqjd,cq->cij", grads, grads, wdet)
    mass = np.einsum("qi,qj,cq->cij", values, values, wdet)
    return stiffness, mass


def boundary_mass_p2(lengths: np.ndarray) -> np.ndarray:
    """Quadratic edge mass L/30 [[4, 2, -1], [2, 16, 2], [-1, 2, 4]] for (end, midpoint, end)
    dofs (adtlert/fem/boundary.py:37-40)."""

    return lengths[:, None, None] * (np.array([[4.0, 2.0, -1.0], [2.0, 16.0, 2.0], [-1.0, 2.0, 4.0]]) / 30.0)[None]


def boundary_mass(lengths: np.ndarray) -> np.ndarray:
    """Linear edge mass L/6 [[2, 1], [1, 2]] (adtlert/fem/boundary.py:31-34)."""

    return lengths[:, None, None] * (np.array([[2.0, 1.0], [1.0, 2.0]]) / 6.0)[None]


def robin_coefficients(centers, normals, surface_mask, surface_level, source, wavenumbers):
    """Mixed-boundary geometry k [(r1.n/|r1|) K1(k|r1|) + (r2.n/|r2|) K1(k|r2|)] / [K0(k|r1|) + K0(k|r2|)]
    for a source at the electrode centroid and its image mirrored at the mean surface level; zero
    on the ground surface (adtlert/fem/boundary.py:43-82). Returns (W, Nb)."""

    image = np.array([source[0], 2.0 * surface_level - source[1]])
    r1, r2 = centers - source, centers - image
    a1, a2 = np.linalg.norm(r1, axis=1), np.linalg.norm(r2, axis=1)
    c1 = np.sum(r1 * normals, axis=1) / np.where(a1 > 0, a1, 1.0)
    c2 = np.sum(r2 * normals, axis=1) / np.where(a2 > 0, a2, 1.0)
    valid = (a1 > 1e-12) & (a2 > 1e-12) & ~surface_mask
    out = np.zeros((len(wavenumbers), len(centers)))
    for w, k in enumerate(wavenumbers):
        den = k0(a1[valid] * k) + k0(a2[valid] * k)
        num = c1[valid] * k1(a1[valid] * k) + c2[valid] * k1(a2[valid] * k)
        stable = den > 1e-12
        row = np.zeros(valid.sum())
        row[stable] = k * num[stable] / den[stable]
        out[w, valid] = row
    return out


def analytic_primary(nodes, cells, positions, source_nodes, wavenumbers) -> np.ndarray:
    """Unit-resistivity half-space primary field (W, E, N): K0(k r)/pi for a surface source,
    (K0(k r) + K0(k r'))/(2 pi) with the mirrored image for a buried one; at the electrode's
    own node K0(k r_nn / 6)/pi with r_nn the nearest-neighbour distance
    (adtlert/forward/ert2p5d.py:78-94, 438-468)."""

    surface = float(nodes[:, 1].max())
    W, E, N = len(wavenumbers), len(positions), len(nodes)
    out = np.zeros((W, E, N))
    for e, (src, node) in enumerate(zip(positions, source_nodes)):
        r = np.linalg.norm(nodes - src, axis=1)
        on_surface = abs(src[1] - surface) <= 1e-8
        if on_surface:
            valid = r > 1e-12
            out[:, e, valid] = k0(np.outer(wavenumbers, r[valid])) / np.pi
        else:
            r2 = np.linalg.norm(nodes - np.array([src[0], 2.0 * surface - src[1]]), axis=1)
            valid = (r > 1e-12) & (r2 > 1e-12)
            out[:, e, valid] = (k0(np.outer(wavenumbers, r[valid])) + k0(np.outer(wavenumbers, r2[valid]))) / (2.0 * np.pi)
        if node >= 0:
            touching = np.unique(cells[(cells == node).any(axis=1)])
            neighbours = touching[touching != node]
            if neighbours.size:
                radius = np.min(np.linalg.norm(nodes[neighbours] - nodes[node], axis=1))
                out[:, e, node] = k0(radius * ELECTRODE_RADIUS_FRACTION * wavenumbers) / np.pi
            else:
                out[:, e, node] = 0.0
    return out
