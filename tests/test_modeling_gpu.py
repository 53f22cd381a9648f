"""GPU check of log_response_and_jacobian (d log rhoa / d log rho, adtlert/forward/modeling.py:
137-162) against the same chain rule applied to the reference's own float64 outputs."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, ERTForward3D, Mesh, Mesh3D, Survey, log_response_and_jacobian
from cases import case3d_inputs, case_inputs
from conftest import ROOT, assert_close

pytestmark = pytest.mark.gpu


def _expected(golden, sigma):
    rhoa = golden["apparent_resistivity"]
    return np.log(rhoa), golden["geometric_factors"][:, None] * golden["jacobian"] * (-sigma[None, :]) / rhoa[:, None]


@pytest.mark.parametrize("name", ["tri_flat", "quad_terrain"])
def test_log_jacobian_2p5d(name):
    inputs = case_inputs(name)
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"], surface_node_ids=inputs.get("surface_node_ids"))
    forward = ERTForward2p5D(mesh, Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    golden = np.load(ROOT / "tests" / "golden" / f"{name}_float64.npz")
    sigma = inputs["sigma"]
    log_rhoa, jacobian = log_response_and_jacobian(forward, torch.as_tensor(sigma, dtype=forward.dtype))
    assert log_rhoa.dtype == np.float64 and jacobian.dtype == np.float64
    expected_log, expected_jacobian = _expected(golden, sigma)
    assert_close(log_rhoa, expected_log, 1e-4, "log rhoa")
    assert_close(jacobian, expected_jacobian, 1e-4, "log-space jacobian")
    ids = inputs.get("parameter_ids")
    if ids is not None:
        count = int(ids.max()) + 1
        chain = np.linspace(0.005, 0.02, count)
        _, aggregated = log_response_and_jacobian(forward, torch.as_tensor(sigma, dtype=forward.dtype), chain=chain,
                                                  jacobian_cell_parameter_ids=ids, jacobian_parameter_count=count)
        rhoa = golden["apparent_resistivity"]
        expected = golden["geometric_factors"][:, None] * golden["jacobian_parameters"] * (-chain[None]) / rhoa[:, None]
        assert_close(aggregated, expected, 1e-4, "aggregated log-space jacobian")


def test_log_jacobian_3d():
    inputs = case3d_inputs("tet_relief")
    forward = ERTForward3D(Mesh3D.from_arrays(inputs["nodes"], inputs["cells"]),
                           Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    golden = np.load(ROOT / "tests" / "golden" / "tet_relief_float64.npz")
    sigma = inputs["sigma"]
    log_rhoa, jacobian = log_response_and_jacobian(forward, torch.as_tensor(sigma, dtype=torch.float32))
    expected_log, expected_jacobian = _expected(golden, sigma)
    assert_close(log_rhoa, expected_log, 1e-4, "log rhoa")
    assert_close(jacobian, expected_jacobian, 1e-4, "log-space jacobian")
