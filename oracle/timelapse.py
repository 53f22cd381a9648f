"""CPU restatement of AD-TLERT's windowed time-lapse Gauss-Newton inversion (TEST
INFRASTRUCTURE ONLY: the checker of the device driver, never part of the product).

Follows, for the configuration of the reference's 363-window example (log-resistivity state,
weighted log L2 misfit, first-order spatial and first-order temporal smoothness in "model" mode,
Gauss-Newton with CGLS, grid line search, model bounds):

* windows and their combination: adtlert/inversion/core.py:433-577;
* the Gauss-Newton loop: core.py:81-300 (linearize, stacked system, candidate, line search,
  chi2, step norm and stop rules);
* the data system: objective.py:56-80 and misfit.py:75-123 (rows W J, rhs -W (pred - obs));
* the regularization blocks: terms.py:75-186 and regularization.py:97-357 (sqrt(lambda) R per
  step, sqrt(lambda_t) first difference in time, rhs -M m);
* CGLS: optimizers.py:314-360 (r kept and s = A^T r recomputed each iteration);
* the line search: objective.py:168-192;
* the log Jacobian: forward/modeling.py:137-162, here from the FP64 oracle operator.

Stacked vectors are time-major (step 0's cells first), the reference's Fortran-order flattening
of its (cells, steps) arrays.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

from .ert2p5d import Oracle2p5D


def neighbour_pairs(nodes, cells):
    """Cells sharing an edge and the |z| part of the edge normal (regularization.py:97-120)."""

    owners: dict[tuple[int, int], list[int]] = {}
    for cell_id, cell in enumerate(np.asarray(cells, dtype=np.int64)):
        for i in range(len(cell)):
            edge = tuple(sorted((int(cell[i]), int(cell[(i + 1) % len(cell)]))))
            owners.setdefault(edge, []).append(cell_id)
    pairs, normal_z = [], []
    for edge, owned in owners.items():
        if len(owned) != 2:
            continue
        tangent = np.asarray(nodes, dtype=float)[edge[1]] - np.asarray(nodes, dtype=float)[edge[0]]
        normal = np.asarray((-tangent[1], tangent[0]))
        length = float(np.linalg.norm(normal))
        if length > 0.0:
            pairs.append(owned)
            normal_z.append(abs(float(normal[-1])) / length)
    return np.asarray(pairs, dtype=np.int64), np.asarray(normal_z)


def roughness_matrix(nodes, cells, z_weight: float = 1.0) -> sp.csr_matrix:
    """First-order constraint matrix R (regularization.py:123-141)."""

    pairs, normal_z = neighbour_pairs(nodes, cells)
    weights = 1.0 + normal_z * (float(z_weight) - 1.0)
    rows = np.repeat(np.arange(len(pairs)), 2)
    data = np.column_stack((weights, -weights)).reshape(-1)
    return sp.coo_matrix((data, (rows, pairs.reshape(-1))), shape=(len(pairs), len(cells))).tocsr()


def temporal_matrix(cells: int, steps: int) -> sp.csr_matrix:
    """First difference in time applied to every cell (regularization.py:302-355)."""

    stencil = np.eye(steps)[1:] - np.eye(steps)[:-1]
    return sp.kron(sp.csr_matrix(stencil), sp.eye(cells, format="csr"), format="csr")


def cgls(matrix: sp.csr_matrix, rhs: np.ndarray, iterations: int, tolerance: float) -> np.ndarray:
    """CGLS for min ||A x - b|| (optimizers.py:314-360), float64, with the same torch CSR
    products and dot products as the reference runs: truncated at 60 iterations on these systems,
    CGLS is sensitive to rounding (two float64 implementations that differ only in summation
    order agree to 1e-14 after 20 iterations but only to ~1e-2 after 60), so the oracle repeats
    the reference's operations to be pinned to it."""

    import torch

    def csr(m):
        return torch.sparse_csr_tensor(torch.as_tensor(m.indptr), torch.as_tensor(m.indices),
                                       torch.as_tensor(m.data, dtype=torch.float64), size=m.shape)

    system, transpose = csr(matrix.tocsr()), csr(matrix.T.tocsr())
    r = torch.as_tensor(np.asarray(rhs).ravel(), dtype=torch.float64)
    x = torch.zeros(system.shape[1], dtype=torch.float64)
    s = transpose @ r
    p = s.clone()
    gamma = torch.dot(s, s)
    gamma0 = float(gamma)
    if gamma0 <= 0.0 or float(torch.dot(r, r)) <= 0.0:
        return x.numpy()
    for _ in range(int(iterations)):
        q = system @ p
        denominator = torch.dot(q, q)
        if float(denominator) <= 0.0:
            break
        alpha = gamma / denominator
        x = x + alpha * p
        r = r - alpha * q
        s = transpose @ r
        gamma_new = torch.dot(s, s)
        if float(gamma_new) <= 0.0 or float(gamma_new) / gamma0 < tolerance:
            break
        p = s + (gamma_new / gamma) * p
        gamma = gamma_new
    return x.numpy().astype(float)


def line_search_tau(state, step, predicted, candidate_predicted, matrix, reference, data_phi) -> float:
    """Grid line search on tau in [0, 1] (objective.py:168-192)."""

    def phi(tau, values):
        roughness = matrix @ (state + tau * step) - reference
        return data_phi(values) + float(roughness @ roughness)

    best_phi = phi(0.0, predicted)
    if phi(1.0, candidate_predicted) < best_phi:
        return 1.0
    best_tau, direction = 0.0, candidate_predicted - predicted
    for index in range(1, 101):
        tau = 0.01 * index
        value = phi(tau, predicted + tau * direction)
        if value < best_phi:
            best_phi, best_tau = value, tau
    return 0.03 if 0.0 < best_tau < 0.03 else best_tau


class OracleTimeLapse:
    """The windowed inversion on the FP64 oracle operator."""

    def __init__(self, nodes, cells, electrodes, measurements, *, max_iterations=15, data_std=0.05,
                 regularization=50.0, temporal_regularization=10.0, z_weight=1.0, model_bounds=(0.001, 1.0e4),
                 step_length=1.0, line_search=True, step_tolerance=1.0e-4, cgls_max_iterations=60,
                 cgls_tolerance=1.0e-12):
        self.operator = Oracle2p5D(nodes, cells, electrodes, measurements)
        self.cells = len(cells)
        self.roughness = roughness_matrix(nodes, cells, z_weight)
        self.max_iterations, self.data_std = int(max_iterations), float(data_std)
        self.regularization, self.temporal = float(regularization), float(temporal_regularization)
        self.log_bounds = None if model_bounds is None else (math.log(model_bounds[0]), math.log(model_bounds[1]))
        self.step_length, self.line_search = float(step_length), bool(line_search)
        self.step_tolerance = float(step_tolerance)
        self.cgls_iterations, self.cgls_tolerance = int(cgls_max_iterations), float(cgls_tolerance)

    def clip(self, state):
        return state if self.log_bounds is None else np.clip(state, *self.log_bounds)

    def linearize(self, log_model):
        """log rhoa and d log rhoa / d log rho of one log model (modeling.py:137-162)."""

        sigma = 1.0 / np.exp(log_model)
        apparent = self.operator.apparent_resistivity(sigma)
        J = self.operator.normal_jacobian(sigma) * self.operator.geometric_factors()[:, None]
        return np.log(apparent), J * (-sigma)[None, :] / apparent[:, None]

    def blocks(self, state, steps):
        """Scaled regularization blocks (matrix, rhs) at the stacked state (terms.py:75-186)."""

        out = []
        if self.regularization > 0.0:
            matrix = math.sqrt(self.regularization) * sp.block_diag([self.roughness] * steps, format="csr")
            out.append((matrix, -(matrix @ state)))
        if self.temporal > 0.0:
            matrix = math.sqrt(self.temporal) * temporal_matrix(self.cells, steps)
            out.append((matrix, -(matrix @ state)))
        return out

    def invert_window(self, observed, initial):
        """(final log models (T, C), predicted (T, D), chi2 history, taus) of one window."""

        steps = observed.shape[0]
        weight = np.full(observed.shape, 1.0 / self.data_std)
        models = self.clip(np.asarray(initial, dtype=float).copy())

        def linearize(states):
            rows = [self.linearize(states[t]) for t in range(steps)]
            return np.vstack([r[0] for r in rows]), [r[1] for r in rows]

        def data_phi(values):
            residual = (values.reshape(observed.shape) - observed) * weight
            return float(np.dot(residual.ravel(), residual.ravel()))

        predicted, jacobians = linearize(models)
        chi2, taus = [], []
        for _ in range(self.max_iterations):
            current = models.reshape(-1)
            blocks = self.blocks(current, steps)
            data = sp.block_diag([sp.csr_matrix(J * weight[t][:, None]) for t, J in enumerate(jacobians)], format="csr")
            rhs = -((predicted - observed) * weight).ravel()
            matrix = sp.vstack([data] + [m for m, _ in blocks], format="csr")
            delta = cgls(matrix, np.concatenate([rhs] + [r for _, r in blocks]), self.cgls_iterations,
                         self.cgls_tolerance)
            candidate = self.clip(models + self.step_length * delta.reshape(models.shape))
            candidate_predicted, candidate_jacobians = linearize(candidate)
            step = candidate.reshape(-1) - current
            tau = 1.0
            if self.line_search:
                objective = sp.vstack([m for m, _ in blocks], format="csr")
                reference = np.concatenate([m @ current + r for m, r in blocks])
                tau = line_search_tau(current, step, predicted.ravel(), candidate_predicted.ravel(), objective,
                                      reference, data_phi)
                step = tau * step
            taus.append(tau)
            if tau < 0.95:
                models = self.clip((current + step).reshape(models.shape))
                predicted, jacobians = linearize(models)
            else:
                models, predicted, jacobians = candidate, candidate_predicted, candidate_jacobians
            chi2.append(float(np.mean(((predicted - observed) * weight) ** 2)))
            if float(np.linalg.norm(step) / max(math.sqrt(current.size), 1.0)) < self.step_tolerance:
                break
        return models, predicted, chi2, taus

    def run(self, observed, initial, window_size=3, window_step=1):
        """Final log models (S, C) as the mean over windows, and per-window chi2 histories."""

        steps = observed.shape[0]
        starts = sorted(set(list(range(0, steps - window_size + 1, max(1, window_step))) + [steps - window_size]))
        contributions = [[] for _ in range(steps)]
        histories = []
        for start in starts:
            models, _, chi2, _ = self.invert_window(observed[start:start + window_size],
                                                    initial[start:start + window_size])
            for offset in range(window_size):
                contributions[start + offset].append(models[offset])
            histories.append(chi2)
        final = np.stack([np.mean(np.column_stack(items), axis=1) for items in contributions])
        return final, histories
