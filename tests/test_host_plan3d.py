"""CPU checks of 3D plans (tetrahedra, Robin faces, Dirichlet dofs, field columns): the device
tables are replayed in NumPy as the kernels index them and compared with the 3D oracle and the
reference's golden outputs."""

import numpy as np
import pytest
import scipy.sparse as sp

from adtlert_b200 import Survey
from adtlert_b200.ert3d import build_problem_3d
from adtlert_b200.geometry3d import Mesh3D
from cases import CASES3D, case3d_inputs
from conftest import ROOT, assert_close
from host_plan import HostPlan, replay_assembly, replay_factor, replay_factor_tiled, replay_solve, replay_solve_tiled
from oracle.ert3d import Oracle3D


@pytest.fixture(scope="module", params=list(CASES3D))
def case(request):
    inputs = case3d_inputs(request.param)
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    problem = build_problem_3d(mesh, survey, inputs["boundary"], element_order=inputs["order"])
    hp = HostPlan(problem.struct())
    assert hp.status == 0, hp.error
    oracle = Oracle3D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"],
                      boundary_mode=inputs["boundary"], element_order=inputs["order"])
    golden = np.load(ROOT / "tests" / "golden" / f"{request.param}_float64.npz")
    return inputs, mesh, problem, hp, oracle, golden


def _values(hp, problem, sigma, identity=True):
    a = problem.arrays
    return replay_assembly(hp, sigma, a["stiffness"], a["mass"], a["bmass"], a["bcoef"][0], a["bcells"], 0.0,
                           identity=identity)


def test_mesh_metadata_matches_the_oracle(case):
    inputs, mesh, problem, hp, oracle, _ = case
    assert np.array_equal(mesh.boundary_faces, oracle.faces)
    assert np.array_equal(mesh.surface_face_mask, oracle.surface_mask)
    assert mesh.is_flat_surface == oracle.flat
    assert np.array_equal(np.sort(problem.fixed), np.sort(oracle.fixed))
    assert np.array_equal(np.sort(hp.fixed), np.sort(hp.iperm[problem.fixed]))
    # stiffness rank 3 (P1) or 9 (P2: constants in the null space); P2 level sets may be wider than
    # the shared-memory solver's 64 and go to the tiled one
    assert hp.R == (3 if inputs["order"] == 1 else 9)
    assert hp.max_m <= 64 or (inputs["order"] == 2 and hp.tiled)


def test_routed_assembly_equals_the_oracle_operator(case):
    inputs, mesh, problem, hp, oracle, _ = case
    ours = sp.csr_matrix((_values(hp, problem, inputs["sigma"]), (hp.csr_row, hp.csr_col)), shape=(hp.N, hp.N))
    expected = oracle.assemble(inputs["sigma"])[hp.perm][:, hp.perm]
    assert_close(ours.toarray(), expected.toarray(), 1e-12, "assembly")
    tangent = sp.csr_matrix((_values(hp, problem, inputs["direction"], identity=False), (hp.csr_row, hp.csr_col)),
                            shape=(hp.N, hp.N))
    expected = oracle.assemble(inputs["direction"], fixed_diagonal=False)[hp.perm][:, hp.perm]
    assert_close(tangent.toarray(), expected.toarray(), 1e-12, "tangent assembly")


def _static_rhs(hp, problem):
    """rhs [N][E'] in solver order as adt_set_static_rhs builds it."""

    unit = sp.csr_matrix((_values(hp, problem, np.ones(problem.counts["C"])), (hp.csr_row, hp.csr_col)),
                         shape=(hp.N, hp.N))
    E = problem.counts["E"]
    rhs = np.zeros((hp.N, E))
    if problem.unit_primary is not None:
        rhs += unit @ problem.unit_primary[0].T[hp.perm]
    if problem.direct is not None:
        rhs += problem.direct[0].T[hp.perm]
    rhs[hp.fixed] = 0.0
    return rhs


def test_replayed_fields_give_the_reference_outputs(case):
    inputs, mesh, problem, hp, oracle, golden = case
    factor, solve = (replay_factor_tiled, replay_solve_tiled) if hp.tiled else (replay_factor, replay_solve)
    factors = factor(hp, _values(hp, problem, inputs["sigma"]))
    fields = solve(hp, factors, _static_rhs(hp, problem))  # [N][E'] solver order
    current, receiver, _ = oracle.fields(inputs["sigma"])
    assert_close(fields[:, problem.current_columns].T, current[:, hp.perm], 1e-10, "current fields")
    assert_close(fields[:, problem.receiver_columns].T, receiver[:, hp.perm], 1e-10, "receiver fields")
    # potential table and transfers exactly as potentials_kernel / transfers_kernel index them
    E = problem.counts["E"]
    K = problem.arrays["cell_dofs"].shape[1]
    rd, rw = hp.rcv_dofs.reshape(E, K), hp.rcv_w.reshape(E, K)
    table = np.zeros((E + 1, E + 1))
    table[:E, :E] = np.einsum("rk,rke->er", rw, fields[rd])
    a, b, m, n = problem.arrays["abmn"].T
    normal = table[a, m] - table[b, m] - table[a, n] + table[b, n]
    assert_close(normal, golden["resistance"], 1e-10, "resistance")
    # Gram Jacobian from the plan's features (the contraction of jacobian_kernel)
    feats = hp.features.reshape(problem.counts["C"], hp.R, K).astype(float)
    x = fields[hp.cdofs.reshape(-1, K)]  # [C][K][E']
    F = np.einsum("cfk,cke->cfe", feats, x)
    G = np.zeros((problem.counts["C"], E + 1, E + 1))
    G[:, :E, :E] = np.einsum("cfe,cfg->ceg", F, F)
    J = -(G[:, m, a] - G[:, m, b] - G[:, n, a] + G[:, n, b]).T
    assert_close(J, golden["jacobian"], 2e-6, "jacobian (float32 template factors)")
