"""CPU checks of the tiled solver used for level sets wider than 64 dofs: its work items are
replayed in NumPy exactly as the kernels index them (every access bounds-checked, every launch
checked for items that write what another item reads or writes) and the result is compared with
a sparse LU solve."""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from adtlert_b200 import Mesh, Survey, synthetic
from adtlert_b200.ert2p5d import build_problem
from adtlert_b200.ert3d import build_problem_3d
from adtlert_b200.geometry3d import Mesh3D
from cases import box_tetrahedra, structured_section
from conftest import assert_close
from host_plan import SMS, HostPlan, panel_splits, replay_assembly, replay_factor_tiled, replay_solve_tiled


def _section_plan():
    xs = np.linspace(0.0, 40.0, 81)
    depths = np.concatenate((np.linspace(0.0, 10.0, 41), np.linspace(10.5, 30.0, 30)))
    nodes, cells = structured_section(xs, depths)
    electrodes = np.column_stack((np.linspace(4.0, 36.0, 17), np.zeros(17)))
    mesh = Mesh.from_arrays(nodes, cells)
    survey = Survey.from_arrays(electrodes, synthetic.dipole_dipole(17, 2, 4))
    problem = build_problem(mesh, survey)
    rng = np.random.default_rng(5)
    sigma = np.exp(rng.normal(np.log(0.01), 0.5, mesh.cell_count))
    a = problem.arrays
    values = replay_assembly(HostPlan(problem.struct()), sigma, problem.stiffness, problem.mass,
                             problem.boundary_mass, problem.robin[3], a["bcells"], problem.wavenumbers[3] ** 2)
    return problem, values


def _box_plan(boundary):
    nodes, cells = box_tetrahedra(nx=9, ny=8, nz=8)
    mesh = Mesh3D.from_arrays(nodes, cells)
    top = np.flatnonzero(np.isclose(nodes[:, 2], 0.0) & np.isclose(nodes[:, 1], 6.0))
    electrodes = nodes[top[np.argsort(nodes[top, 0])]]
    survey = Survey.from_arrays(electrodes, np.asarray([(0, 1, 3, 4), (1, 2, 5, 6), (2, -1, 4, 5)]))
    problem = build_problem_3d(mesh, survey, boundary)
    rng = np.random.default_rng(6)
    sigma = np.exp(rng.normal(np.log(0.01), 0.5, mesh.cell_count))
    a = problem.arrays
    values = replay_assembly(HostPlan(problem.struct()), sigma, a["stiffness"], a["mass"], a["bmass"],
                             a["bcoef"][0], a["bcells"], 0.0)
    return problem, values


@pytest.mark.parametrize("build", [_section_plan, lambda: _box_plan("mixed"), lambda: _box_plan("dirichlet")],
                         ids=["section", "box-mixed", "box-dirichlet"])
def test_tiled_factor_and_solve_match_a_sparse_lu(build):
    problem, values = build()
    hp = HostPlan(problem.struct())
    assert hp.status == 0, hp.error
    assert hp.tiled == 1 and hp.max_m > 64, "the case must exercise the tiled solver"
    A = sp.csr_matrix((values, (hp.csr_row, hp.csr_col)), shape=(hp.N, hp.N)).tocsc()
    rhs = np.random.default_rng(0).standard_normal((hp.N, 70))
    expected = spl.splu(A).solve(rhs)
    # panels split over 2-8 depth ranges (few tiles per launch on 148 SMs), and never split
    splits = {panel_splits(len(hp.titems.reshape(-1, 4)[b:e]), 1)
              for b, e in hp.tranges.reshape(-1, 2)[3 * hp.levels:]}
    assert max(splits) > 1
    for sms in (SMS, 1):
        factors = replay_factor_tiled(hp, values, sms=sms)
        assert_close(replay_solve_tiled(hp, factors, rhs), expected, 1e-9, f"tiled solve ({sms} SMs)")


def test_tiled_items_cover_every_tile_once():
    problem, _ = _section_plan()
    hp = HostPlan(problem.struct())
    L = hp.levels
    items = hp.titems.reshape(-1, 4)
    for level in range(L):
        t0, t1 = hp.level_begin[level], hp.level_begin[level + 1]
        b, e = hp.tranges[2 * (2 * L + level)], hp.tranges[2 * (2 * L + level) + 1]
        tiles = {(int(t), int(i)) for t, i, _, _ in items[b:e]}
        expected = {(t, i) for t in range(t0, t1) for i in range(-(-int(hp.tasks[t][1]) // 64))}
        assert tiles == expected
        b, e = hp.tranges[2 * level], hp.tranges[2 * level + 1]
        for t in range(t0, t1):
            rows = sorted((int(r0), int(n)) for tt, r0, n, _ in items[b:e] if tt == t)
            assert rows[0][0] == 0 and sum(n for _, n in rows) == int(hp.tasks[t][1])
