"""GPU parity of the 2.5D operator against the reference's golden vectors and the FP64 oracle.

Every product is checked with the reference test suite's metric (max-norm relative error,
adtlert tests/test_forward_gpu.py:18-27) at the float32 tolerance of 1e-4, against (a) the
reference's own float32 outputs on identical inputs and (b) the float64 oracle; relational
checks (half-space, scaling, dot tests, finite differences, reciprocity, repeatability) follow
the reference's tests.
"""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, apparent_resistivity_autograd, synthetic
from cases import FLAT_CASES, case_inputs
from conftest import ROOT, assert_close
from oracle.ert2p5d import Oracle2p5D

pytestmark = pytest.mark.gpu

TOL = 1e-4  # float32 parity bar (max-norm relative)


@pytest.fixture(scope="module", params=FLAT_CASES)
def case(request):
    name = request.param
    inputs = case_inputs(name)
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = ERTForward2p5D.from_mesh_survey(mesh, survey)
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
    both(forward.wavenumbers, "wavenumbers", g32, g64, 1e-6)
    both(forward.weights, "weights", g32, g64, 1e-6)
    # the reference evaluates the half-space factors in float32; ours are float64 rounded to float32
    both(forward._geometric_factors(), "geometric_factors", g32, g64, 1e-5)
    both(response.apparent_resistivity, "apparent_resistivity", g32, g64)
    both(response.resistance, "resistance", g32, g64)
    both(response.electrode_potentials, "electrode_potentials", g32, g64)
    homogeneous = forward.apparent_resistivity_values(torch.full((forward.C,), 0.01))
    both(homogeneous, "homogeneous_apparent_resistivity", g32, g64)
    # the reference itself is within 2.6e-3 of 100 ohm-m on this coarse test section
    assert_close(homogeneous, np.full(forward.D, 100.0), 5e-3, "half-space")


def test_fields_match_the_oracle(case):
    name, inputs, forward, g32, g64 = case
    fields = forward._fields(torch.as_tensor(inputs["sigma"], dtype=torch.float32)).total.cpu().numpy()
    order = forward._dof_order
    expected = g64["total_fields"][:, :, order].transpose(0, 2, 1)  # (W, N, E) in solver order
    assert_close(fields, expected, TOL, "total fields")


def test_normal_jacobian_matches_the_reference(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    J = forward.jacobian(sigma)
    assert J.shape == (forward.D, forward.C) and J.device.type == "cpu" and J.dtype == torch.float32
    both(J, "jacobian", g32, g64)
    assert torch.equal(forward.jacobian(sigma, batch_size=7), J)
    if "jacobian_parameters" in g32.files:
        ids = inputs["parameter_ids"]
        _, aggregated = forward.solve_with_jacobian(sigma, jacobian_cell_parameter_ids=ids,
                                                    jacobian_parameter_count=int(ids.max()) + 1)
        both(aggregated, "jacobian_parameters", g32, g64)


def test_exact_jacobian_matches_the_reference(case):
    name, inputs, forward, g32, g64 = case
    if "jacobian_exact" not in g32.files:
        pytest.skip("case without the exact-derivative Jacobian")
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    exact = forward.jacobian(sigma, include_robin_boundary_derivative=True, normal_sensitivity=False)
    both(exact, "jacobian_exact", g32, g64)


def test_matrix_free_products_match_the_reference(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    cotangent = torch.as_tensor(inputs["cotangent"], dtype=torch.float32)
    direction = torch.as_tensor(inputs["direction"], dtype=torch.float32)
    both(forward.vjp(sigma, cotangent), "vjp", g32, g64)
    both(forward.jvp(sigma, direction), "jvp", g32, g64)
    both(forward.normal_vjp(sigma, cotangent), "normal_vjp", g32, g64)
    both(forward.normal_jvp(sigma, direction), "normal_jvp", g32, g64)
    if "normal_vjp_parameters" in g32.files:
        ids = inputs["parameter_ids"]
        both(forward.normal_vjp(sigma, cotangent, cell_parameter_ids=ids, parameter_count=int(ids.max()) + 1),
             "normal_vjp_parameters", g32, g64)


def test_dot_tests_and_jacobian_consistency(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    rng = np.random.default_rng(7)
    direction = torch.as_tensor(rng.standard_normal(forward.C) * inputs["sigma"] * 1e-2, dtype=torch.float32)
    cotangent = torch.as_tensor(rng.standard_normal(forward.D), dtype=torch.float32)
    lhs = float((forward.jvp(sigma, direction).double() * cotangent.double()).sum())
    rhs = float((direction.double() * forward.vjp(sigma, cotangent).double()).sum())
    assert lhs == pytest.approx(rhs, rel=1e-4)
    J = forward.jacobian(sigma).double()
    assert_close(J.T @ cotangent.double(), forward.normal_vjp(sigma, cotangent), TOL, "J^T c")
    assert_close(J @ direction.double(), forward.normal_jvp(sigma, direction), TOL, "J d")


def test_jvp_matches_finite_differences(case):
    name, inputs, forward, g32, g64 = case
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    rng = np.random.default_rng(3)
    direction = torch.as_tensor(rng.standard_normal(forward.C), dtype=torch.float32) * sigma
    h = 1e-3
    numeric = (forward.resistance(sigma + h * direction).double() - forward.resistance(sigma - h * direction).double()) / (2 * h)
    assert_close(forward.jvp(sigma, direction), numeric, 5e-3, "jvp vs central differences")


def test_scaling_and_reciprocity():
    inputs = case_inputs("tri_flat")
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = ERTForward2p5D.from_mesh_survey(mesh, survey)
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    base = forward.apparent_resistivity_values(sigma)
    assert_close(forward.apparent_resistivity_values(sigma / 3.0), 3.0 * base, 1e-5, "1/sigma scaling")
    assert_close(forward.apparent_resistivity_values(sigma, currents=2.0), base / 2.0, 1e-6, "1/I scaling")
    swapped = Survey.from_arrays(inputs["electrodes"], inputs["measurements"][:, [2, 3, 0, 1]])
    other = ERTForward2p5D.from_mesh_survey(mesh, swapped)
    assert_close(other.resistance(sigma), forward.resistance(sigma), 1e-5, "reciprocity")


def test_kernels_are_repeatable_and_follow_the_current_stream():
    inputs = case_inputs("quad_flat")
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                                              Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    first = forward.jacobian(sigma)
    assert all(torch.equal(first, forward.jacobian(sigma)) for _ in range(5))
    forward.close()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        on_stream = forward.jacobian(sigma)
    stream.synchronize()
    assert torch.equal(on_stream, first)
    gradient = forward.vjp(sigma, torch.ones(forward.D))
    assert all(torch.equal(gradient, forward.vjp(sigma, torch.ones(forward.D))) for _ in range(3))


def test_series_batching_cache_and_factorization_reuse():
    inputs = case_inputs("tri_flat")
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    reference = ERTForward2p5D.from_mesh_survey(mesh, survey)
    forward = ERTForward2p5D.from_mesh_survey(mesh, survey, series_batch_steps=2)
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    series = torch.stack([sigma, sigma * 1.2, sigma * 0.8])
    rng = np.random.default_rng(5)
    cotangents = torch.as_tensor(rng.standard_normal((3, forward.D)), dtype=torch.float32)
    resistance = torch.stack([reference.resistance(m) for m in series])
    gradient = torch.stack([reference.vjp(m, c) for m, c in zip(series, cotangents)])
    assert_close(forward.resistance_series(series), resistance, 1e-6, "series resistance")
    before = forward._solver.factorizations
    assert_close(forward.vjp_series(series, cotangents), gradient, 1e-5, "series vjp")
    assert forward._solver.factorizations == before  # the adjoint batches reuse the forward factorizations
    forward.resistance_series(series * 1.7)
    after = forward._solver.factorizations
    assert after == before + 2
    assert_close(forward.vjp_series(series, cotangents), gradient, 1e-5, "series vjp after eviction")
    assert forward._solver.factorizations == after + 2  # stale factorizations are not reused
    hits = forward.normal_field_cache_info()["hits"]
    forward.normal_vjp_series(series, torch.ones(3, forward.D))
    assert forward.normal_field_cache_info()["hits"] >= hits + 3


def test_autograd_bridge_matches_vjp():
    inputs = case_inputs("tri_flat")
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                                              Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float64).clone().requires_grad_()
    current = torch.tensor(1.5, dtype=torch.float64, requires_grad=True)
    weights = torch.as_tensor(np.random.default_rng(2).standard_normal(forward.D))
    rhoa = apparent_resistivity_autograd(sigma, forward, current)
    assert rhoa.dtype == torch.float64
    (rhoa * weights).sum().backward()
    scale = forward._geometric_factors().double() / 1.5
    assert_close(sigma.grad, forward.vjp(sigma.detach().float(), (weights * scale).float()), 1e-5, "autograd vjp")
    expected = -float((weights * rhoa.detach()).sum()) / 1.5
    assert float(current.grad) == pytest.approx(expected, rel=1e-5)
    series = torch.stack([sigma.detach(), sigma.detach() * 1.3]).float().requires_grad_()
    out = apparent_resistivity_autograd(series, forward)
    assert out.shape == (2, forward.D)
    out.sum().backward()
    assert series.grad.shape == series.shape


def test_validation_errors():
    inputs = case_inputs("tri_flat")
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    with pytest.raises(ValueError, match="topographic_geometric_factor_mode"):
        ERTForward2p5D.from_mesh_survey(mesh, survey, topographic_geometric_factor_mode="x")
    with pytest.raises(ValueError, match="non-negative"):
        ERTForward2p5D.from_mesh_survey(mesh, survey, normal_field_cache_max_entries=-1)
    forward = ERTForward2p5D.from_mesh_survey(mesh, survey)
    with pytest.raises(ValueError, match="conductivity must be scalar"):
        forward.solve(torch.ones(3))
    with pytest.raises(ValueError, match="positive"):
        forward.solve(-torch.ones(forward.C))
    with pytest.raises(ValueError, match="parameter_count requires"):
        forward.normal_vjp(torch.ones(forward.C), torch.ones(forward.D), parameter_count=3)
    with pytest.raises(ValueError, match="batch_size"):
        forward.jacobian(torch.ones(forward.C), batch_size=0)
    first = forward.resistance(torch.ones(forward.C))
    forward.close()
    assert torch.equal(forward.resistance(torch.ones(forward.C)), first)


def test_flat_benchmark_section_matches_the_oracle():
    """The benchmark workload itself: apparent resistivity and sampled Jacobian rows vs FP64."""

    nodes, cells, electrodes, rows = synthetic.flat_section()
    sigma = synthetic.layered_model(nodes, cells, seed=0)
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    oracle = Oracle2p5D(nodes, cells, electrodes, rows)
    rhoa = forward.apparent_resistivity_values(torch.as_tensor(sigma))
    expected = oracle.apparent_resistivity(sigma.astype(float))
    assert_close(rhoa, expected, TOL, "flat section apparent resistivity")
    J = forward.jacobian(torch.as_tensor(sigma)).numpy()
    picks = np.arange(0, len(rows), 97)
    sub = Oracle2p5D(nodes, cells, electrodes, rows[picks])
    assert_close(J[picks], sub.normal_jacobian(sigma.astype(float)), TOL, "flat section jacobian rows")
    assert forward.kernel_launches() > 0


def test_non_finite_fields_raise_and_are_not_cached():
    # a subnormal conductivity puts the float32 fields beyond the float32 range
    inputs = case_inputs("tri_flat")
    forward = ERTForward2p5D(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                             Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    tiny = torch.full((forward.C,), 1e-40)
    for _ in range(2):  # the second call solves again instead of serving cached fields
        with pytest.raises(FloatingPointError, match="total fields"):
            forward.jacobian(tiny)
    assert forward.normal_field_cache_info()["entries"] == 0
    with pytest.raises(FloatingPointError, match="total fields"):
        forward.solve(tiny)
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    assert torch.isfinite(forward.jacobian(sigma)).all()


def test_fused_forward_substitution_gives_the_two_phase_fields():
    from adtlert_b200 import _native
    nodes, cells, electrodes, abmn = synthetic.flat_section()
    forward = ERTForward2p5D(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, abmn))
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 4), dtype=torch.float32).cuda()[None].contiguous()
    other = sigma.clone()
    slot, stream = forward._solver.lookup(1)["slot"], forward._stream()

    def fields(factorize, solve_sigma):
        out = torch.full((1, forward.W, forward.N, forward.E), float("nan"), device="cuda")
        if factorize:
            forward._call(factorize, slot, _native.ptr(sigma), 1, stream)
        forward._call("adt_solve_fields", slot, _native.ptr(solve_sigma), 1, _native.ptr(out), stream)
        return out.cpu().double()

    two_phase = fields("adt_factorize", sigma)
    fused = fields("adt_factorize_fields", sigma)
    again = fields(None, sigma)            # reduced right-hand sides consumed: the full solve
    forward._call("adt_factorize_fields", slot, _native.ptr(sigma), 1, stream)
    elsewhere = fields(None, other)        # another sigma buffer: the full solve
    for name, value in (("fused", fused), ("again", again), ("elsewhere", elsewhere)):
        assert torch.isfinite(value).all()
        assert_close(value, two_phase, 1e-6, f"{name} fields vs factorize + solve_fields")


def test_one_call_forward_and_jacobian_entry_points():
    """adt_forward / adt_jacobian equal the step-by-step calls they compose, bitwise."""

    from adtlert_b200 import _native

    nodes, cells, electrodes, rows = synthetic.flat_section()
    forward = ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    W, N, E, D, C = forward.W, forward.N, forward.E, forward.D, forward.C
    models = torch.as_tensor(np.stack([synthetic.layered_model(nodes, cells, s) for s in (4, 5)]), device="cuda")
    handle = forward._stream()

    def run(name, *args):
        forward._call(name, *args)

    fields = torch.empty((2, W, N, E), device="cuda")
    normal = torch.empty((2, D), dtype=torch.float64, device="cuda")
    recip = torch.empty_like(normal)
    run("adt_forward", 14, _native.ptr(models), 2, _native.ptr(fields), _native.ptr(normal), _native.ptr(recip), handle)
    fields2, normal2, recip2 = torch.empty_like(fields), torch.empty_like(normal), torch.empty_like(recip)
    run("adt_factorize_fields", 13, _native.ptr(models), 2, handle)
    run("adt_solve_fields", 13, _native.ptr(models), 2, _native.ptr(fields2), handle)
    run("adt_measure", _native.ptr(fields2), 2, _native.ptr(normal2), _native.ptr(recip2), None, handle)
    assert torch.equal(fields, fields2) and torch.equal(normal, normal2) and torch.equal(recip, recip2)

    one = models[1]
    J = torch.empty((D - 10, C), device="cuda")
    run("adt_jacobian", 14, _native.ptr(one), _native.ptr(fields[0]), 10, D - 10, _native.ptr(J), handle)
    expected = torch.empty_like(J)
    run("adt_normal_jacobian", _native.ptr(fields2[1]), 10, D - 10, _native.ptr(expected), handle)
    assert torch.equal(J, expected)
