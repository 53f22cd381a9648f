"""The 3D oracle (oracle/ert3d.py) against the reference's own 3D outputs (tests/golden/tet_*)."""

import numpy as np
import pytest

from cases import CASES3D, case3d_inputs
from conftest import ROOT, assert_close
from oracle.ert3d import Oracle3D


@pytest.fixture(scope="module", params=list(CASES3D))
def pinned(request):
    inputs = case3d_inputs(request.param)
    golden = np.load(ROOT / "tests" / "golden" / f"{request.param}_float64.npz")
    oracle = Oracle3D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"],
                      boundary_mode=inputs["boundary"], element_order=inputs["order"])
    return request.param, inputs, golden, oracle


def test_forward_products(pinned):
    _, inputs, golden, oracle = pinned
    sigma = inputs["sigma"]
    assert_close(oracle.geometric_factors(), golden["geometric_factors"], 1e-12)
    assert_close(oracle.resistance(sigma), golden["resistance"], 1e-11)
    assert_close(oracle.apparent_resistivity(sigma), golden["apparent_resistivity"], 1e-11)
    current = oracle.fields(sigma)[0]
    assert_close(current, golden["node_potentials"][oracle.cur_ids], 1e-11)
    homogeneous = oracle.apparent_resistivity(np.full(len(sigma), 0.01))
    assert_close(homogeneous, golden["homogeneous_apparent_resistivity"], 1e-11)


def test_derivative_products(pinned):
    _, inputs, golden, oracle = pinned
    sigma, g, d = inputs["sigma"], inputs["cotangent"], inputs["direction"]
    assert_close(oracle.jacobian(sigma), golden["jacobian"], 1e-11)
    assert_close(oracle.jacobian(sigma, True), golden["jacobian_robin"], 1e-11)
    assert_close(oracle.vjp(sigma, g), golden["vjp"], 1e-11)
    assert_close(oracle.jvp(sigma, d), golden["jvp"], 1e-11)
    assert_close(oracle.normal_vjp(sigma, g), golden["normal_vjp"], 1e-11)
    assert_close(oracle.normal_jvp(sigma, d), golden["normal_jvp"], 1e-11)


def test_reference_float32_is_within_the_parity_bar_of_float64(pinned):
    name, _, golden, _ = pinned
    single = np.load(ROOT / "tests" / "golden" / f"{name}_float32.npz")
    for key in ("resistance", "apparent_resistivity", "jacobian", "vjp", "jvp"):
        assert_close(single[key], golden[key], 1e-4)
