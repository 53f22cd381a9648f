"""Host pieces of the device Gauss-Newton driver on CPU: the neighbour lists of the smoothing
operator, the line search on the objective's quadratic, and the window starts, each against the
oracle restatement of the reference (oracle/timelapse.py)."""

import numpy as np
import scipy.sparse as sp

from adtlert_b200 import synthetic
from adtlert_b200.timelapse import line_search_tau, neighbour_graph, window_starts
from cases import case_inputs
from oracle import timelapse as oracle


def _laplacian(ptr, cells, w2, count):
    rows = np.repeat(np.arange(count), np.diff(ptr))
    off = sp.coo_matrix((-w2, (rows, cells)), shape=(count, count)).tocsr()
    return off + sp.diags(np.asarray(-off.sum(axis=1)).ravel())


def test_neighbour_lists_give_the_roughness_normal_operator():
    for z_weight in (1.0, 0.3):
        for nodes, cells in ((case_inputs("tri_flat")["nodes"], case_inputs("tri_flat")["cells"]),
                             synthetic.flat_section()[:2]):
            R = oracle.roughness_matrix(nodes, cells, z_weight)
            ptr, nbr, w2 = neighbour_graph(nodes, cells, z_weight)
            L = _laplacian(ptr, nbr, w2, len(cells))
            assert abs(L - (R.T @ R)).max() < 1e-12


def test_quadratic_line_search_matches_the_grid_search():
    rng = np.random.default_rng(4)
    for trial in range(200):
        n, m = 30, 20
        state, step = rng.standard_normal(n), rng.standard_normal(n) * rng.uniform(0.01, 3)
        matrix = sp.csr_matrix(rng.standard_normal((m, n)) * rng.uniform(0.1, 2))
        predicted, observed = rng.standard_normal(40), rng.standard_normal(40)
        candidate = predicted + rng.standard_normal(40) * rng.uniform(0.1, 5)

        def data_phi(values):
            return float(np.sum((values - observed) ** 2))

        expected = oracle.line_search_tau(state, step, predicted, candidate, matrix, np.zeros(m), data_phi)
        r0, r1 = predicted - observed, candidate - predicted
        ms, mm = matrix @ step, matrix @ state
        got = line_search_tau((r0 @ r0 + mm @ mm, r0 @ r1 + mm @ ms, r1 @ r1 + ms @ ms))
        assert got == expected, (trial, got, expected)


def test_window_starts():
    assert window_starts(365, 3) == list(range(363))
    assert window_starts(10, 3, 4) == [0, 4, 7]
