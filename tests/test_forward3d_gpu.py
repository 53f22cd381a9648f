"""GPU parity of the 3D operator against the reference's golden vectors and the FP64 3D oracle.

Every product is compared with the reference's own float32 and float64 outputs on identical
inputs (max-norm relative error, bar 1e-4); the relational checks follow the reference's 3D tests
(dot tests, finite differences, the autograd bridge, series batching).
"""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward3D, Mesh3D, Survey, apparent_resistivity_autograd
from cases import CASES3D, case3d_inputs
from conftest import ROOT, assert_close
from oracle.ert3d import Oracle3D

pytestmark = pytest.mark.gpu

TOL = 1e-4  # float32 parity bar (max-norm relative)


@pytest.fixture(scope="module", params=list(CASES3D))
def case(request):
    name = request.param
    inputs = case3d_inputs(name)
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = ERTForward3D.from_mesh_survey(mesh, survey, boundary_mode=inputs["boundary"],
                                            element_order=inputs["order"])
    golden32 = np.load(ROOT / "tests" / "golden" / f"{name}_float32.npz")
    golden64 = np.load(ROOT / "tests" / "golden" / f"{name}_float64.npz")
    return name, inputs, forward, golden32, golden64


def both(actual, key, golden32, golden64, tol=TOL):
    e32 = assert_close(actual, golden32[key], tol, f"{key} vs reference float32")
    e64 = assert_close(actual, golden64[key], tol, f"{key} vs reference float64")
    return e32, e64


def test_forward_matches_the_reference(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    response = forward.solve(sigma)
    assert response.apparent_resistivity.device.type == "cpu"
    assert response.apparent_resistivity.dtype == torch.float32
    both(forward._geometric_factors(), "geometric_factors", g32, g64, 1e-5 if "relief" not in name else TOL)
    both(response.apparent_resistivity, "apparent_resistivity", g32, g64)
    both(response.resistance, "resistance", g32, g64)
    used = forward._current_electrode_ids
    nodes = response.node_potentials.numpy()
    assert np.isnan(np.delete(nodes, used, axis=0)).all()
    assert_close(nodes[used], g64["node_potentials"][used], TOL, "node potentials")
    homogeneous = forward.apparent_resistivity_values(torch.full((forward.C,), 0.01))
    both(homogeneous, "homogeneous_apparent_resistivity", g32, g64)


def test_jacobians_match_the_reference(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    J = forward.jacobian(sigma, batch_size=5)
    assert J.device.type == "cpu" and J.dtype == torch.float32 and J.shape == (forward.D, forward.C)
    both(J, "jacobian", g32, g64)
    both(forward.jacobian(sigma, include_robin_boundary_derivative=True), "jacobian_robin", g32, g64)


def test_matrix_free_products_match_the_reference(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    g = torch.as_tensor(inputs["cotangent"], dtype=torch.float32)
    d = torch.as_tensor(inputs["direction"], dtype=torch.float32)
    both(forward.vjp(sigma, g), "vjp", g32, g64)
    both(forward.jvp(sigma, d), "jvp", g32, g64)
    both(forward.normal_vjp(sigma, g), "normal_vjp", g32, g64)
    both(forward.normal_jvp(sigma, d), "normal_jvp", g32, g64)


def test_dot_tests_and_jacobian_consistency(case):
    name, inputs, forward, *_ = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    rng = np.random.default_rng(3)
    d = torch.as_tensor(rng.standard_normal(forward.C) * inputs["sigma"] * 1e-2, dtype=torch.float32)
    g = torch.as_tensor(rng.standard_normal(forward.D), dtype=torch.float32)
    exact = forward.jacobian(sigma, include_robin_boundary_derivative=True).double()
    normal = forward.jacobian(sigma).double()
    assert_close(forward.jvp(sigma, d), exact @ d.double(), TOL, "J_robin d")
    assert_close(forward.vjp(sigma, g), exact.T @ g.double(), TOL, "J_robin^T g")
    assert_close(forward.normal_jvp(sigma, d), normal @ d.double(), TOL, "J d")
    assert_close(forward.normal_vjp(sigma, g), normal.T @ g.double(), TOL, "J^T g")


def test_jvp_matches_finite_differences(case):
    name, inputs, forward, *_ = case
    sigma = inputs["sigma"]
    direction = inputs["direction"] / np.abs(inputs["direction"]).max() * sigma.min() * 1e-1
    oracle = Oracle3D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"],
                      boundary_mode=inputs["boundary"], element_order=inputs["order"])
    h = 1e-3
    fd = (oracle.resistance(sigma + h * direction) - oracle.resistance(sigma - h * direction)) / (2 * h)
    ours = forward.jvp(torch.as_tensor(sigma, dtype=torch.float32), torch.as_tensor(direction, dtype=torch.float32))
    assert_close(ours, fd, 1e-3, "jvp vs central differences of the oracle")


def test_series_cache_and_parameter_aggregation():
    inputs = case3d_inputs("tet_mixed")
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = ERTForward3D(mesh, survey, series_batch_steps=2, normal_field_cache_max_entries=4)
    base = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    series = torch.stack([base, base * 1.5, base * 0.5])
    together = forward.resistance_series(series)
    for step in range(3):
        assert_close(together[step], forward.resistance(series[step]), 1e-6, "series vs single")
    # conductivity scaling: R(c sigma) = R(sigma) / c
    assert_close(together[1] * 1.5, together[0], 1e-5, "scaling")
    info = forward.normal_field_cache_info()
    assert info["hits"] >= 3 and info["entries"] <= 4
    ids = np.arange(forward.C) // 6
    ids[::7] = -1
    count = int(ids.max()) + 1
    J = forward.jacobian(base).numpy()
    aggregated = forward.jacobian(base, jacobian_cell_parameter_ids=ids, jacobian_parameter_count=count).numpy()
    expected = np.zeros((forward.D, count))
    for c in np.flatnonzero(ids >= 0):
        expected[:, ids[c]] += J[:, c]
    assert_close(aggregated, expected, 1e-5, "parameter aggregation")
    g = np.random.default_rng(4).standard_normal(forward.D)
    fused = forward.normal_vjp(base, torch.as_tensor(g, dtype=torch.float32), cell_parameter_ids=ids,
                               parameter_count=count)
    assert_close(fused, expected.T @ g, 1e-4, "fused normal_vjp aggregation")


def test_autograd_bridge_matches_vjp():
    inputs = case3d_inputs("tet_relief")
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = ERTForward3D(mesh, survey)
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32).requires_grad_(True)
    rhoa = apparent_resistivity_autograd(sigma, forward)
    g = torch.as_tensor(inputs["cotangent"], dtype=torch.float32)
    (rhoa * g).sum().backward()
    expected = forward.vjp(sigma.detach(), g * forward._geometric_factors())
    assert_close(sigma.grad, expected, 1e-6, "autograd gradient")
    assert_close(rhoa.detach(), forward.apparent_resistivity_values(sigma.detach()), 1e-6, "autograd forward")


def test_validation_errors():
    inputs = case3d_inputs("tet_mixed")
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    with pytest.raises(ValueError):
        ERTForward3D(mesh, survey, boundary_mode="neumann")
    with pytest.raises(ValueError):
        ERTForward3D(mesh, survey, geometric_factor_mode="exact")
    with pytest.raises(ValueError):
        ERTForward3D(mesh, Survey.from_arrays(inputs["electrodes"][:, :2], inputs["measurements"]))
    forward = ERTForward3D(mesh, survey)
    with pytest.raises(ValueError):
        forward.jacobian(torch.ones(forward.C), batch_size=0)
    with pytest.raises(ValueError):
        forward.resistance(torch.ones(forward.C - 1))
