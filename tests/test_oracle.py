"""The oracle against the reference's own golden vectors (CPU only)."""

import numpy as np
import pytest

from cases import FLAT_CASES, case_inputs
from conftest import ROOT, assert_close
from oracle import baseline
from oracle.ert2p5d import Oracle2p5D, inverse_cosine_weights, wavenumber_bounds

GOLDEN = ROOT / "tests" / "golden"


@pytest.fixture(scope="module", params=FLAT_CASES)
def pinned(request):
    name = request.param
    inputs = case_inputs(name)
    oracle = Oracle2p5D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])
    return name, inputs, oracle, np.load(GOLDEN / f"{name}_float64.npz")


def test_quadrature_and_geometric_factors(pinned):
    name, inputs, oracle, golden = pinned
    k, w = inverse_cosine_weights(*wavenumber_bounds(inputs["electrodes"]))
    assert_close(k, golden["wavenumbers"], 1e-14, "wavenumbers")
    assert_close(w, golden["weights"], 1e-14, "weights")
    assert_close(oracle.geometric_factors(), golden["geometric_factors"], 1e-14, "geometric factors")
    assert oracle.nnz == int(golden["nnz"])


def test_forward_products(pinned):
    name, inputs, oracle, golden = pinned
    sigma = inputs["sigma"]
    assert_close(oracle.fields(sigma)[1], golden["total_fields"], 1e-11, "fields")
    assert_close(oracle.apparent_resistivity(sigma), golden["apparent_resistivity"], 1e-12, "rhoa")
    assert_close(oracle.resistance(sigma), golden["resistance"], 1e-12, "resistance")
    assert_close(oracle.apparent_resistivity(np.full(oracle.C, 0.01)), golden["homogeneous_apparent_resistivity"], 1e-12, "half-space")


def test_derivative_products(pinned):
    name, inputs, oracle, golden = pinned
    sigma, cot, direction = inputs["sigma"], inputs["cotangent"], inputs["direction"]
    assert_close(oracle.normal_jacobian(sigma), golden["jacobian"], 1e-12, "jacobian")
    assert_close(oracle.vjp(sigma, cot), golden["vjp"], 1e-12, "vjp")
    assert_close(oracle.jvp(sigma, direction), golden["jvp"], 1e-12, "jvp")
    assert_close(oracle.normal_vjp(sigma, cot), golden["normal_vjp"], 1e-12, "normal vjp")
    assert_close(oracle.normal_jvp(sigma, direction), golden["normal_jvp"], 1e-12, "normal jvp")
    if "jacobian_exact" in golden.files:
        assert_close(oracle.exact_jacobian(sigma), golden["jacobian_exact"], 1e-12, "exact jacobian")
    if "jacobian_parameters" in golden.files:
        ids = inputs["parameter_ids"]
        assert_close(oracle.normal_jacobian(sigma, ids), golden["jacobian_parameters"], 1e-12, "parameter jacobian")
        assert_close(oracle.normal_vjp(sigma, cot, ids), golden["normal_vjp_parameters"], 1e-12, "parameter vjp")


def test_c_contraction_matches_the_oracle_einsum(pinned):
    name, inputs, oracle, golden = pinned
    assert_close(baseline.jacobian(oracle, inputs["sigma"], threads=3), golden["jacobian"], 1e-12, "C contraction")


def test_reference_float32_is_within_the_parity_bar_of_float64(pinned):
    """What the reference itself achieves in float32 (the scale of the 1e-4 parity bar)."""

    name, inputs, oracle, golden = pinned
    g32 = np.load(GOLDEN / f"{name}_float32.npz")
    for key in ("apparent_resistivity", "jacobian", "vjp", "jvp", "normal_vjp", "normal_jvp"):
        assert_close(g32[key], golden[key], 1e-4, f"reference float32 {key}")
