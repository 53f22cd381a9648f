"""The 3D operator on a survey shaped like the 3D benchmark one: a 12 x 8 electrode grid, every
electrode a current and a receiver electrode, so 188 field columns with singularity removal
(more than the 64 of the tensor-core Jacobian; the FP32 Gram kernel takes up to 200). Checked
against the FP64 oracle on the resistances and on a row subset of the Jacobian, and by dot tests
on the whole Jacobian (max-norm relative, bar 1e-4)."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward3D, Mesh3D, Survey
from cases import grid_survey_3d
from conftest import assert_close
from oracle.ert3d import Oracle3D

pytestmark = pytest.mark.gpu

TOL = 1e-4


def test_grid_survey_with_188_field_columns():
    g = grid_survey_3d()
    forward = ERTForward3D(Mesh3D.from_arrays(g["nodes"], g["cells"]), Survey.from_arrays(g["electrodes"], g["measurements"]))
    assert forward.columns == 188
    sigma = torch.as_tensor(g["sigma"], dtype=torch.float32)
    oracle = Oracle3D(g["nodes"], g["cells"], g["electrodes"], g["measurements"])
    assert_close(forward.resistance(sigma), oracle.resistance(g["sigma"]), TOL, "resistance vs oracle")
    J = forward.jacobian(sigma, batch_size=32)
    assert J.shape == (len(g["measurements"]), len(g["cells"])) and torch.isfinite(J).all()
    rows = Oracle3D(g["nodes"], g["cells"], g["electrodes"], g["measurements"][:64])
    assert_close(J[:64], rows.jacobian(g["sigma"]), TOL, "jacobian rows vs oracle")
    rng = np.random.default_rng(5)
    d = torch.as_tensor(rng.standard_normal(forward.C) * g["sigma"] * 1e-2, dtype=torch.float32)
    c = torch.as_tensor(rng.standard_normal(forward.D), dtype=torch.float32)
    assert_close(forward.normal_jvp(sigma, d), J.double() @ d.double(), TOL, "J d")
    assert_close(forward.normal_vjp(sigma, c), J.double().T @ c.double(), TOL, "J^T c")
