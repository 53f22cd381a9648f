"""GPU parity of operators whose level sets are wider than 64 dofs (the tiled solver) against
the FP64 oracles: a deep 2.5D section and a 3D box."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, ERTForward3D, Mesh, Mesh3D, Survey, synthetic
from cases import box_tetrahedra, structured_section
from conftest import assert_close
from oracle.ert2p5d import Oracle2p5D
from oracle.ert3d import Oracle3D

pytestmark = pytest.mark.gpu

TOL = 1e-4


def test_deep_section_uses_the_tiled_solver_and_matches_the_oracle():
    xs = np.linspace(0.0, 40.0, 81)
    depths = np.concatenate((np.linspace(0.0, 10.0, 41), np.linspace(10.5, 30.0, 30)))
    nodes, cells = structured_section(xs, depths)
    electrodes = np.column_stack((np.linspace(4.0, 36.0, 17), np.zeros(17)))
    measurements = synthetic.dipole_dipole(17, 2, 4)
    forward = ERTForward2p5D(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, measurements))
    assert forward.plan_info["max_block"] > 64
    rng = np.random.default_rng(8)
    sigma = np.exp(rng.normal(np.log(0.01), 0.5, len(cells)))
    oracle = Oracle2p5D(nodes, cells, electrodes, measurements)
    s32 = torch.as_tensor(sigma, dtype=torch.float32)
    assert_close(forward.resistance(s32), oracle.resistance(sigma), TOL, "resistance")
    assert_close(forward.jacobian(s32), oracle.normal_jacobian(sigma), TOL, "jacobian")


@pytest.mark.parametrize("boundary", ["mixed", "dirichlet"])
def test_wide_box_uses_the_tiled_solver_and_matches_the_oracle(boundary):
    nodes, cells = box_tetrahedra(nx=9, ny=8, nz=8)
    top = np.flatnonzero(np.isclose(nodes[:, 2], 0.0) & np.isclose(nodes[:, 1], 6.0))
    electrodes = nodes[top[np.argsort(nodes[top, 0])]]
    count = len(electrodes)
    measurements = np.asarray([(i, i + 1, i + 1 + n, i + 2 + n) for n in (1, 2) for i in range(count) if i + 2 + n < count])
    forward = ERTForward3D(Mesh3D.from_arrays(nodes, cells), Survey.from_arrays(electrodes, measurements),
                           boundary_mode=boundary)
    assert forward.plan_info["max_block"] > 64
    rng = np.random.default_rng(9)
    sigma = np.exp(rng.normal(np.log(0.01), 0.5, len(cells)))
    oracle = Oracle3D(nodes, cells, electrodes, measurements, boundary_mode=boundary)
    s32 = torch.as_tensor(sigma, dtype=torch.float32)
    assert_close(forward.resistance(s32), oracle.resistance(sigma), TOL, "resistance")
    assert_close(forward.jacobian(s32, include_robin_boundary_derivative=True),
                 oracle.jacobian(sigma, True), TOL, "jacobian")
    g = rng.standard_normal(len(measurements))
    assert_close(forward.vjp(s32, torch.as_tensor(g, dtype=torch.float32)), oracle.vjp(sigma, g), TOL, "vjp")
