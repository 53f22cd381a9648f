"""FP64 NumPy/SciPy restatement of AD-TLERT's 3D tetrahedral operator (adtlert/forward/ert3d.py).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``): the product never imports this.
Covers element orders 1 and 2, mixed and Dirichlet far-field boundaries, singularity removal on flat
surfaces (point sources otherwise) and analytic or numerical geometric factors. The sparse solve
uses SciPy SuperLU where the reference calls cuDSS.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

ELECTRODE_RADIUS_FRACTION_3D = 0.5  # adtlert/forward/ert3d.py:47-49
_TETRA_FACES = ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1))  # adtlert/mesh/core3d.py:16
_P2_EDGES = ((0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3))  # adtlert/fem/tetrahedron.py:13


def quadratic_dofs(nodes, cells, faces):
    """Edge-midpoint dofs numbered on first use, cell by cell (adtlert/mesh/core.py:27-44,
    core3d.py:211-234): dof coordinates, cell dofs (C x 10), face dofs (F x 6)."""

    points, index = [np.asarray(p, dtype=float) for p in nodes], {}

    def midpoint(a, b):
        key = (min(a, b), max(a, b))
        if key not in index:
            index[key] = len(points)
            points.append(0.5 * (points[key[0]] + points[key[1]]))
        return index[key]

    cell_dofs = [[*c] + [midpoint(c[i], c[j]) for i, j in _P2_EDGES] for c in cells.tolist()]
    face_dofs = [[*f] + [midpoint(f[i], f[j]) for i, j in ((0, 1), (1, 2), (2, 0))] for f in faces.tolist()]
    return np.asarray(points), np.asarray(cell_dofs, dtype=np.int64), np.asarray(face_dofs, dtype=np.int64)


def p2_values(bary):
    """Ten-node shape functions (tetrahedron.py:59-66)."""

    edges = np.stack([4.0 * bary[..., i] * bary[..., j] for i, j in _P2_EDGES], axis=-1)
    return np.concatenate((bary * (2.0 * bary - 1.0), edges), axis=-1)


def p2_stiffness(grads, vol):
    """Ten-node stiffness with the 4-point rule (tetrahedron.py:92-127), grads (C, 4, 3)."""

    a, b = (5.0 + 3.0 * math.sqrt(5.0)) / 20.0, (5.0 - math.sqrt(5.0)) / 20.0
    out = np.zeros((len(vol), 10, 10))
    for q in range(4):
        lam = np.full(4, b)
        lam[q] = a
        vertex = (4.0 * lam - 1.0)[None, :, None] * grads
        edge = np.stack([4.0 * (lam[i] * grads[:, j] + lam[j] * grads[:, i]) for i, j in _P2_EDGES], axis=1)
        g = np.concatenate((vertex, edge), axis=1)
        out += np.einsum("eid,ejd->eij", g, g)
    return out * (vol / 4.0)[:, None, None]


def p2_face_mass(area):
    """Six-node triangle mass matrix by a 7-point degree-5 rule (tetrahedron.py:69-89 uses a
    degree-4 rule; both are exact for the degree-4 products)."""

    s15 = math.sqrt(15.0)
    a1, a2 = (6.0 - s15) / 21.0, (6.0 + s15) / 21.0
    w1, w2 = (155.0 - s15) / 1200.0, (155.0 + s15) / 1200.0
    pts = [(1 / 3, 1 / 3, 1 / 3)]
    wts = [9.0 / 40.0]
    for a, w in ((a1, w1), (a2, w2)):
        for k in range(3):
            p = [a, a, a]
            p[k] = 1.0 - 2.0 * a
            pts.append(tuple(p))
            wts.append(w)
    bary = np.asarray(pts)
    shape = np.concatenate((bary * (2.0 * bary - 1.0),
                            np.stack([4.0 * bary[:, i] * bary[:, j] for i, j in ((0, 1), (1, 2), (2, 0))], 1)), 1)
    return area * np.einsum("q,qi,qj->ij", np.asarray(wts), shape, shape)


def boundary_faces(nodes, cells):
    """Sorted boundary faces, owning cells, centers, areas, outward normals (core3d.py:37-65)."""

    faces = np.sort(cells[:, _TETRA_FACES], axis=-1).reshape(-1, 3)
    unique, first, counts = np.unique(faces, axis=0, return_index=True, return_counts=True)
    keep = counts == 1
    faces, face_cells = unique[keep], first[keep] // 4
    fn = nodes[faces]
    centers = fn.mean(axis=1)
    cross = np.cross(fn[:, 1] - fn[:, 0], fn[:, 2] - fn[:, 0])
    norm = np.linalg.norm(cross, axis=1)
    normals = cross / norm[:, None]
    outward = np.sum(normals * (centers - nodes[cells[face_cells]].mean(axis=1)), axis=1) >= 0.0
    return faces, face_cells, centers, 0.5 * norm, normals * np.where(outward, 1.0, -1.0)[:, None]


def locate(nodes, cells, points, tol=1e-8):
    """Containing tetrahedron and barycentric weights (core3d.py:68-107)."""

    cn = nodes[cells]
    inverse = np.linalg.inv(np.stack([cn[:, i] - cn[:, 0] for i in (1, 2, 3)], axis=-1))
    lower, upper = cn.min(axis=1) - tol, cn.max(axis=1) + tol
    ids, weights = np.full(len(points), -1), np.zeros((len(points), 4))
    for p, point in enumerate(points):
        nearest = int(np.argmin(np.linalg.norm(nodes - point, axis=1)))
        if np.linalg.norm(nodes[nearest] - point) <= tol:
            candidates = np.flatnonzero(np.any(cells == nearest, axis=1))
        else:
            candidates = np.flatnonzero(np.all((point >= lower) & (point <= upper), axis=1))
        for c in candidates:
            local = inverse[c] @ (point - cn[c, 0])
            bary = np.asarray((1.0 - local.sum(), *local))
            if np.all(bary >= -tol) and np.all(bary <= 1.0 + tol):
                bary[np.abs(bary) <= tol] = 0.0
                ids[p], weights[p] = c, bary / bary.sum()
                break
    if np.any(ids < 0):
        raise ValueError("points lie outside the tetrahedral mesh")
    return ids, weights


class Oracle3D:
    """P1 or ten-node P2 tetrahedral DC operator (adtlert/forward/ert3d.py:114-983)."""

    def __init__(self, nodes, cells, electrodes, measurements, boundary_mode="mixed",
                 singularity_removal=True, geometric_factor_mode="auto", element_order=1):
        self.vertices = np.asarray(nodes, dtype=float)
        self.cells = np.asarray(cells, dtype=np.int64)
        self.nodes = self.vertices
        self.electrodes = np.asarray(electrodes, dtype=float)
        self.measurements = np.asarray(measurements, dtype=np.int64)
        self.faces, self.face_cells, centers, areas, normals = boundary_faces(self.vertices, self.cells)
        if element_order == 2:  # ert3d.py:179-193
            self.nodes, self.dofs, face_dofs = quadratic_dofs(self.vertices, self.cells, self.faces)
        else:
            self.dofs, face_dofs = self.cells, self.faces
        K = self.dofs.shape[1]
        self.K = K
        N, C, E = len(self.nodes), len(self.cells), len(self.electrodes)
        self.N, self.C, self.E = N, C, E
        self.surface_mask = normals[:, 2] > 1e-8
        surface_nodes = np.unique(self.faces[self.surface_mask])
        self.surface_level = float(self.nodes[:, 2].max())
        tol = max(1e-8, max(float(np.ptp(self.nodes[:, 2])), 1.0) * 1e-8)
        self.flat = bool(np.ptp(self.nodes[surface_nodes, 2]) <= tol)
        # P1 stiffness templates (fem/tetrahedron.py:37-56)
        cn = self.vertices[self.cells]
        jac = np.stack([cn[:, i] - cn[:, 0] for i in (1, 2, 3)], axis=-1)
        ref = np.asarray(((-1.0, -1.0, -1.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)))
        grads = np.einsum("ij,ejk->eik", ref, np.linalg.inv(jac))
        vol = np.abs(np.linalg.det(jac)) / 6.0
        if element_order == 2:
            self.volume_templates = p2_stiffness(grads, vol)
        else:
            self.volume_templates = vol[:, None, None] * np.einsum("eid,ejd->eij", grads, grads)
        self.cell_templates = self.volume_templates.copy()
        self.boundary_mode = boundary_mode
        if boundary_mode == "mixed":  # ert3d.py:235-266
            center = self.electrodes.mean(axis=0)
            mass = np.asarray(((2.0, 1.0, 1.0), (1.0, 2.0, 1.0), (1.0, 1.0, 2.0))) / 12.0
            for f in np.flatnonzero(~self.surface_mask):
                radial = centers[f] - center
                r2 = float(radial @ radial)
                if r2 <= 0.0:
                    continue
                alpha = max(float(radial @ normals[f]) / r2, 0.0)
                if alpha == 0.0:
                    continue
                c = self.face_cells[f]
                local = [int(np.flatnonzero(self.dofs[c] == n)[0]) for n in face_dofs[f]]
                face_mass = p2_face_mass(areas[f]) if element_order == 2 else areas[f] * mass
                self.cell_templates[c][np.ix_(local, local)] += alpha * face_mass
        # assembly routing (ert3d.py:292-351)
        rows = np.repeat(self.dofs, K, axis=1).reshape(-1)
        cols = np.tile(self.dofs, (1, K)).reshape(-1)
        self.fixed = np.unique(face_dofs[~self.surface_mask].reshape(-1)) if boundary_mode == "dirichlet" else np.zeros(0, int)
        fixed_mask = np.zeros(N, dtype=bool)
        fixed_mask[self.fixed] = True
        self.pair_keep = ~fixed_mask[rows] & ~fixed_mask[cols]
        self.rows, self.cols = rows, cols
        # electrodes used as current and receiver rows (ert3d.py:95-105)
        slots = np.where(self.measurements == -1, E, self.measurements)
        self.cur_ids = np.unique(slots[:, :2][slots[:, :2] < E])
        self.rcv_ids = np.unique(slots[:, 2:][slots[:, 2:] < E])
        cmap = np.full(E + 1, -1)
        cmap[self.cur_ids] = np.arange(len(self.cur_ids))
        cmap[E] = len(self.cur_ids)
        rmap = np.full(E + 1, -1)
        rmap[self.rcv_ids] = np.arange(len(self.rcv_ids))
        rmap[E] = len(self.rcv_ids)
        self.abmn = np.stack((cmap[slots[:, 0]], cmap[slots[:, 1]], rmap[slots[:, 2]], rmap[slots[:, 3]]), 1)
        ids, w = locate(self.vertices, self.cells, self.electrodes)
        if element_order == 2:  # ert3d.py:71-90
            w = p2_values(w)
        self.electrode_matrix = sp.coo_matrix(
            (w.reshape(-1), (np.repeat(np.arange(E), K), self.dofs[ids].reshape(-1))), shape=(E, N)
        ).tocsr()
        self.singularity = singularity_removal and self.flat
        self.use_numerical_gf = geometric_factor_mode == "numerical" or (geometric_factor_mode == "auto" and not self.flat)
        unit = self.assemble(np.ones(C))
        if self.singularity:  # ert3d.py:367-395
            primary = np.stack([self.primary(s) for s in self.electrodes[self.cur_ids]])
            self.source_rhs = (unit @ primary.T).T
        else:
            self.source_rhs = self.electrode_matrix[self.cur_ids].toarray()
        self.receiver_rhs = self.electrode_matrix[self.rcv_ids].toarray()
        if boundary_mode == "dirichlet":
            self.source_rhs[:, self.fixed] = 0.0
            self.receiver_rhs[:, self.fixed] = 0.0

    def primary(self, source):
        """(1/r + 1/r') / (4 pi), r <= 1e-12 replaced by half the nearest distance (ert3d.py:367-385)."""

        mirror = source.copy()
        mirror[2] = 2.0 * self.surface_level - source[2]
        d, dm = np.linalg.norm(self.nodes - source, axis=1), np.linalg.norm(self.nodes - mirror, axis=1)
        fallback = max(float(np.min(d[d > 1e-12])) * ELECTRODE_RADIUS_FRACTION_3D, 1e-12)
        d = np.where(d > 1e-12, d, fallback)
        dm = np.where(dm > 1e-12, dm, fallback)
        return (1.0 / d + 1.0 / dm) / (4.0 * np.pi)

    def assemble(self, sigma, robin=True, fixed_diagonal=True) -> sp.csr_matrix:
        templates = self.cell_templates if robin else self.volume_templates
        vals = (np.asarray(sigma, dtype=float)[:, None, None] * templates).reshape(-1)
        keep = self.pair_keep
        A = sp.coo_matrix((vals[keep], (self.rows[keep], self.cols[keep])), shape=(self.N, self.N)).tocsr()
        if fixed_diagonal and len(self.fixed):
            A = A + sp.coo_matrix((np.ones(len(self.fixed)), (self.fixed, self.fixed)), shape=A.shape)
        return A.tocsr()

    def fields(self, sigma):
        lu = spl.splu(self.assemble(sigma).tocsc())
        current = lu.solve(self.source_rhs.T).T  # (n_cur, N)
        receiver = lu.solve(self.receiver_rhs.T).T  # (n_rcv, N)
        return current, receiver, lu

    def _transfer(self, current):
        P = np.pad(current @ self.electrode_matrix[self.rcv_ids].T.toarray(), ((0, 1), (0, 1)))
        a, b, m, n = self.abmn.T
        return P[a, m] - P[b, m] - P[a, n] + P[b, n]  # ert3d.py:558-566

    def resistance(self, sigma):
        return self._transfer(self.fields(sigma)[0])

    def geometric_factors(self):
        if not self.use_numerical_gf:
            q = self.measurements
            pts = self.electrodes[np.clip(q, 0, None)]
            real = q != -1

            def inv(i, j):
                d = np.linalg.norm(pts[:, i] - pts[:, j], axis=-1)
                return np.where(real[:, i] & real[:, j], 1.0 / np.where(d > 0, d, 1.0), 0.0)

            return 2.0 * math.pi / (inv(0, 2) - inv(0, 3) - inv(1, 2) + inv(1, 3))
        return 1.0 / self.resistance(np.ones(self.C))  # ert3d.py:577-597

    def apparent_resistivity(self, sigma, currents=1.0):
        return self.geometric_factors() * self.resistance(sigma) / currents

    def _pairs(self, cotangent):
        nc, nr = len(self.cur_ids), len(self.rcv_ids)
        p = np.zeros((nc + 1, nr + 1))
        a, b, m, n = self.abmn.T
        g = np.asarray(cotangent, dtype=float)
        np.add.at(p, (a, m), g)
        np.add.at(p, (a, n), -g)
        np.add.at(p, (b, m), -g)
        np.add.at(p, (b, n), g)
        return p[:nc, :nr]

    def _cell_gradient(self, phi, lam, robin):
        T = self.cell_templates if robin else self.volume_templates
        T = np.where(self.pair_keep.reshape(-1, self.K, self.K), T, 0.0)
        return -np.einsum("sci,cij,scj->c", lam[:, self.dofs], T, phi[:, self.dofs])

    def vjp(self, sigma, cotangent):
        current, receiver, lu = self.fields(sigma)
        rhs = self._pairs(cotangent) @ self.receiver_rhs
        lam = lu.solve(rhs.T).T
        return self._cell_gradient(current, lam, robin=True)  # ert3d.py:744-772

    def normal_vjp(self, sigma, cotangent):
        current, receiver, _ = self.fields(sigma)
        return self._cell_gradient(current, self._pairs(cotangent) @ receiver, robin=False)

    def jvp(self, sigma, direction):
        current, _, lu = self.fields(sigma)
        dA = self.assemble(direction, robin=True, fixed_diagonal=False)
        delta = lu.solve(-(dA @ current.T)).T
        return self._transfer(delta)  # ert3d.py:774-793

    def normal_jvp(self, sigma, direction):
        current, receiver, _ = self.fields(sigma)
        dA = self.assemble(direction, robin=False, fixed_diagonal=False)
        gram = np.pad(-(dA @ current.T).T @ receiver.T, ((0, 1), (0, 1)))
        a, b, m, n = self.abmn.T
        return gram[a, m] - gram[b, m] - gram[a, n] + gram[b, n]  # ert3d.py:843-865

    def jacobian(self, sigma, include_robin_boundary_derivative=False):
        current, receiver, _ = self.fields(sigma)
        T = self.cell_templates if include_robin_boundary_derivative else self.volume_templates
        T = np.where(self.pair_keep.reshape(-1, self.K, self.K), T, 0.0)
        cur = np.vstack((current, np.zeros((1, self.N))))
        rcv = np.vstack((receiver, np.zeros((1, self.N))))
        a, b, m, n = self.abmn.T
        u = (cur[a] - cur[b])[:, self.dofs]
        v = (rcv[m] - rcv[n])[:, self.dofs]
        return -np.einsum("dci,cij,dcj->dc", v, T, u)  # ert3d.py:867-927
