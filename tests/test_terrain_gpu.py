"""GPU parity of the 2.5D terrain operator (refined auxiliary fields, numerical primary field,
optional numerical geometric factors) against the reference's own outputs on identical inputs.

The reference computes terrain in float64; its float32 and float64 runs differ by about 1e-5
(float32 geometry and linear templates). Our fields are float32 on the GPU and every product is
held to the 1e-4 max-norm relative bar against both runs."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey
from cases import TERRAIN_CASES, case_inputs
from conftest import ROOT, assert_close

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module", params=TERRAIN_CASES)
def case(request):
    name = request.param
    inputs = case_inputs(name)
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"], surface_node_ids=inputs["surface_node_ids"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = ERTForward2p5D.from_mesh_survey(mesh, survey, topographic_geometric_factor_mode=inputs["gf_mode"])
    golden32 = np.load(ROOT / "tests" / "golden" / f"{name}_float32.npz")
    golden64 = np.load(ROOT / "tests" / "golden" / f"{name}_float64.npz")
    return name, inputs, forward, golden32, golden64


def both(actual, key, golden32, golden64, tol=TOL):
    assert_close(actual, golden32[key], tol, f"{key} vs reference float32")
    return assert_close(actual, golden64[key], tol, f"{key} vs reference float64")


def test_terrain_forward_matches_the_reference(case):
    name, inputs, forward, g32, g64 = case
    assert forward.use_numerical_primary and forward.dtype == torch.float64
    assert forward.use_numerical_geometric_factors == (inputs["gf_mode"] == "numerical")
    assert_close(forward.discretization.dof_nodes, g64["discretization_nodes"], 1e-12, "refined nodes")
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float64)
    response = forward.solve(sigma)
    assert response.resistance.dtype == torch.float64 and response.resistance.device.type == "cpu"
    both(forward._geometric_factors(), "geometric_factors", g32, g64)
    both(response.apparent_resistivity, "apparent_resistivity", g32, g64)
    both(response.resistance, "resistance", g32, g64)
    both(response.electrode_potentials, "electrode_potentials", g32, g64)
    both(response.integrated_potentials, "integrated_potentials", g32, g64)
    homogeneous = forward.apparent_resistivity_values(torch.full((forward.C,), 0.01, dtype=torch.float64))
    both(homogeneous, "homogeneous_apparent_resistivity", g32, g64)


def test_terrain_derivatives_match_the_reference(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float64)
    g = torch.as_tensor(inputs["cotangent"], dtype=torch.float64)
    d = torch.as_tensor(inputs["direction"], dtype=torch.float64)
    J = forward.jacobian(sigma)
    assert J.shape == (forward.D, forward.C) and J.dtype == torch.float64
    both(J, "jacobian", g32, g64)
    both(forward.vjp(sigma, g), "vjp", g32, g64)
    both(forward.jvp(sigma, d), "jvp", g32, g64)
    both(forward.normal_vjp(sigma, g), "normal_vjp", g32, g64)
    both(forward.normal_jvp(sigma, d), "normal_jvp", g32, g64)
    if "jacobian_exact" in g64.files:
        exact = forward.jacobian(sigma, include_robin_boundary_derivative=True, normal_sensitivity=False)
        both(exact, "jacobian_exact", g32, g64)
    ids = inputs.get("parameter_ids")
    if ids is not None:
        count = int(ids.max()) + 1
        _, aggregated = forward.solve_with_jacobian(sigma, jacobian_cell_parameter_ids=ids,
                                                    jacobian_parameter_count=count)
        both(aggregated, "jacobian_parameters", g32, g64)
        fused = forward.normal_vjp(sigma, g, cell_parameter_ids=ids, parameter_count=count)
        both(fused, "normal_vjp_parameters", g32, g64)


def test_terrain_cache_round_trip(tmp_path):
    inputs = case_inputs("tri_terrain")
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"], surface_node_ids=inputs["surface_node_ids"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    first = ERTForward2p5D(mesh, survey, terrain_cache_dir=tmp_path)
    files = sorted(tmp_path.glob("*.npz"))
    assert len(files) == 1
    second = ERTForward2p5D(mesh, survey, terrain_cache_dir=tmp_path)
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float64)
    assert torch.equal(first.resistance(sigma), second.resistance(sigma))
