"""CPU checks of the plan builder: ordering, routing, elimination schedule, template factors.

The solver and assembly tables are replayed in NumPy exactly as the CUDA kernels index them,
so these tests also bound every device access of a plan before it runs on a GPU.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from adtlert_b200 import Mesh, Survey, synthetic
from adtlert_b200.ert2p5d import build_problem
from cases import FLAT_CASES, case_inputs
from conftest import assert_close
from host_plan import HostPlan, replay_assembly, replay_backward, replay_factor, replay_solve
from oracle.ert2p5d import Oracle2p5D


def _plan(nodes, cells, electrodes, measurements):
    mesh = Mesh.from_arrays(nodes, cells)
    survey = Survey.from_arrays(electrodes, measurements)
    problem = build_problem(mesh, survey)
    hp = HostPlan(problem.struct())
    assert hp.status == 0, hp.error
    return mesh, survey, problem, hp


@pytest.fixture(scope="module", params=FLAT_CASES)
def case(request):
    inputs = case_inputs(request.param)
    mesh, survey, problem, hp = _plan(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])
    oracle = Oracle2p5D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])
    return inputs, problem, hp, oracle


def test_ordering_is_a_block_tridiagonal_permutation(case):
    inputs, problem, hp, oracle = case
    assert sorted(hp.perm.tolist()) == list(range(hp.N))
    assert np.array_equal(hp.iperm[hp.perm], np.arange(hp.N))
    assert hp.nnz == oracle.nnz and hp.max_m <= 64
    block = np.empty(hp.N, dtype=int)
    offsets = sorted({(int(t[2]), int(t[1])) for t in hp.tasks})
    for b, (off, m) in enumerate(offsets):
        block[off:off + m] = b
    rows = hp.csr_row
    assert np.all(np.abs(block[rows] - block[hp.csr_col]) <= 1), "coupling beyond neighbouring levels"


def test_routed_assembly_equals_the_oracle_operator(case):
    inputs, problem, hp, oracle = case
    sigma = inputs["sigma"]
    reference = oracle.assemble(sigma)
    for w in (0, len(problem.wavenumbers) - 1):
        values = replay_assembly(hp, sigma, problem.stiffness, problem.mass, problem.boundary_mass,
                                 problem.robin[w], problem.arrays["bcells"], problem.wavenumbers[w] ** 2)
        ours = sp.csr_matrix((values, (hp.csr_row, hp.csr_col)), shape=(hp.N, hp.N))
        expected = oracle.matrix(reference[w]).tocsr()[hp.perm][:, hp.perm]
        assert_close(ours.toarray(), expected.toarray(), 1e-12, "assembly")


def test_replayed_block_cyclic_reduction_solves_the_system(case):
    inputs, problem, hp, oracle = case
    values = replay_assembly(hp, inputs["sigma"], problem.stiffness, problem.mass, problem.boundary_mass,
                             problem.robin[0], problem.arrays["bcells"], problem.wavenumbers[0] ** 2)
    factors = replay_factor(hp, values)
    A = sp.csr_matrix((values, (hp.csr_row, hp.csr_col)), shape=(hp.N, hp.N)).tocsc()
    rhs = np.random.default_rng(0).standard_normal((hp.N, 7))
    expected = spl.splu(A).solve(rhs)
    assert_close(replay_solve(hp, factors, rhs), expected, 1e-10, "solve")
    # forward substitution fused into the Schur-update launches, then the backward levels alone
    fused, reduced = replay_factor(hp, values, rhs)
    assert np.array_equal(fused, factors, equal_nan=True)
    assert_close(replay_backward(hp, fused, reduced), expected, 1e-10, "fused forward + backward")


def test_template_factors_reproduce_the_templates(case):
    inputs, problem, hp, oracle = case
    K = problem.stiffness.shape[1]
    feats = hp.features.reshape(-1, hp.R, K).astype(float)
    for w in (0, 5):
        scale = hp.fscale.reshape(-1, hp.R)[w].astype(float)
        F = feats * scale[None, :, None]
        gram = np.einsum("cfi,cfj->cij", F, F)
        expected = problem.weights[w] * (problem.stiffness + problem.wavenumbers[w] ** 2 * problem.mass)
        assert_close(gram, expected, 2e-6, "template factors")


def test_pair_and_receiver_routings_match_the_oracle_scatter(case):
    inputs, problem, hp, oracle = case
    E, D = oracle.E, len(oracle.measurements)
    rng = np.random.default_rng(1)
    normal, recip = rng.standard_normal(D), rng.standard_normal(D)
    pairs = np.zeros((E, E))
    for e in range(E):
        for f in range(E):
            slot = e * (E + 1) + f
            acc = 0.0
            for code in hp.pair_list[hp.pair_ptr[slot]:hp.pair_ptr[slot + 1]]:
                d, kind = code >> 2, code & 3
                value = normal[d] if kind < 2 else recip[d]
                acc += -value if kind & 1 else value
            pairs[e, f] = acc
    assert_close(pairs, oracle._pair_cotangent(normal, recip), 1e-14, "pair scatter")
    rhs = np.zeros((hp.N, E))
    for i, dof in enumerate(hp.rdof_dof):
        for j in range(hp.rdof_ptr[i], hp.rdof_ptr[i + 1]):
            rhs[dof] += pairs[:, hp.rdof_rcv[j]] * hp.rdof_w[j]
    assert_close(rhs, (pairs @ oracle.electrode_matrix).T[hp.perm], 1e-14, "adjoint rhs routing")


def test_flat_benchmark_section_plan():
    nodes, cells, electrodes, rows = synthetic.flat_section()
    mesh, survey, problem, hp = _plan(nodes, cells, electrodes, rows)
    assert (hp.N, hp.nnz) == (4961, 34081) and hp.max_m <= 41
    assert hp.levels == int(np.ceil(np.log2(hp.nb))) + 1
    assert hp.R == 5  # rank-2 stiffness + rank-3 mass of a P1 triangle
    values = replay_assembly(hp, np.full(mesh.cell_count, 0.01), problem.stiffness, problem.mass,
                             problem.boundary_mass, problem.robin[0], problem.arrays["bcells"], problem.wavenumbers[0] ** 2)
    factors = replay_factor(hp, values)
    A = sp.csr_matrix((values, (hp.csr_row, hp.csr_col)), shape=(hp.N, hp.N)).tocsc()
    rhs = np.random.default_rng(2).standard_normal((hp.N, 3))
    assert_close(replay_solve(hp, factors, rhs), spl.splu(A).solve(rhs), 1e-9, "flat section solve")


def test_invalid_problems_are_rejected():
    inputs = case_inputs("tri_flat")
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    problem = build_problem(mesh, survey)
    problem.arrays["abmn"][0, 0] = 99
    hp = HostPlan(problem.struct())
    assert hp.status == 1 and "measurement slots" in hp.error
