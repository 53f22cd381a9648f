"""The 2.5D terrain configuration at full size (40,000 triangles under a three-sinusoid surface,
96 electrodes, 2538 rows, numerical geometric factors, 19 wavenumbers): the derivative checks the
configuration names, through the public API.

* dot test: <g, jvp(s, d)> = <vjp(s, g), d> for the exact resistance derivatives;
* central differences with h = 1e-3 in log conductivity on 32 seeded directions against jvp
  (adtlert/forward/ert2p5d.py:873-890);
* the normal-quadrupole Jacobian applied to a direction equals normal_jvp (ert2p5d.py:914-943).
"""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def terrain():
    nodes, cells, surface, electrodes, rows = synthetic.terrain_section()
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(nodes, cells, surface_node_ids=surface),
                                              Survey.from_arrays(electrodes, rows),
                                              topographic_geometric_factor_mode="numerical")
    sigma = torch.as_tensor(synthetic.correlated_model(nodes, cells, 0))
    assert (forward.C, forward.D, forward.E, forward.W) == (40000, 2538, 96, 19)
    return forward, sigma


def test_dot_test(terrain):
    forward, sigma = terrain
    rng = np.random.default_rng(1)
    g = torch.as_tensor(rng.standard_normal(forward.D))
    d = sigma * torch.as_tensor(rng.standard_normal(forward.C) * 1e-2, dtype=torch.float32)
    left = float(torch.dot(g.double(), forward.jvp(sigma, d).double()))
    right = float(torch.dot(forward.vjp(sigma, g).double(), d.double()))
    assert abs(left - right) <= 1e-5 * max(abs(left), abs(right))


def test_central_differences_in_log_conductivity_on_32_directions(terrain):
    forward, sigma = terrain
    rng = np.random.default_rng(2)
    h = 1e-3
    worst = 0.0
    for _ in range(32):
        direction = rng.standard_normal(forward.C)
        direction /= np.linalg.norm(direction) / np.sqrt(forward.C)  # unit RMS in log conductivity
        step = torch.as_tensor(np.exp(h * direction), dtype=torch.float32)
        plus = forward.resistance(sigma * step).double()
        minus = forward.resistance(sigma / step).double()
        fd = (plus - minus) / (2 * h)
        exact = forward.jvp(sigma, sigma * torch.as_tensor(direction, dtype=torch.float32)).double()
        worst = max(worst, float(torch.linalg.norm(fd - exact) / torch.linalg.norm(exact)))
    assert worst < 2e-3, worst


def test_normal_jacobian_matches_normal_jvp(terrain):
    forward, sigma = terrain
    d = sigma * torch.as_tensor(np.random.default_rng(3).standard_normal(forward.C) * 1e-2, dtype=torch.float32)
    J = forward.jacobian(sigma)
    assert J.shape == (forward.D, forward.C) and torch.isfinite(J).all()
    applied = J.double() @ d.double()
    reference = forward.normal_jvp(sigma, d).double()
    assert float(torch.linalg.norm(applied - reference) / torch.linalg.norm(reference)) < 1e-5
