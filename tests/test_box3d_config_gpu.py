"""The 3D configuration at full size against the FP64 oracle (adtlert/forward/ert3d.py:114-983):
244,800 P1 tetrahedra, 45,018 nodes, 12 x 8 surface electrodes, 4000 dipole-dipole rows, mixed
boundary, singularity removal. The oracle's SuperLU fields take seconds here, so parity is
checked directly on 64 rows spread over the survey: resistances and Jacobian rows within the
1e-4 float32 bar (max-norm relative), plus the row-range Jacobian call against the full one.
"""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward3D, Mesh3D, Survey, _native, synthetic
from conftest import assert_close
from oracle.ert3d import Oracle3D

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def box():
    nodes, cells = synthetic.box_section()
    electrodes, rows = synthetic.grid_survey()
    sigma = synthetic.ellipsoid_model(nodes, cells, 0)
    forward = ERTForward3D(Mesh3D.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows),
                           series_batch_steps=1)
    sample = np.linspace(0, len(rows) - 1, 64).astype(int)
    oracle = Oracle3D(nodes, cells, electrodes, rows[sample])
    fields = oracle.fields(sigma.astype(float))
    oracle.fields = lambda s: fields  # one SuperLU solve serves both comparisons
    return forward, torch.as_tensor(sigma), oracle, sample


def test_resistances_match_the_oracle(box):
    forward, sigma, oracle, sample = box
    ours = forward.resistance(sigma).numpy()[sample]
    assert_close(ours, oracle.resistance(sigma.numpy().astype(float)), 1e-4, "3D box resistances")


def test_jacobian_rows_match_the_oracle(box):
    forward, sigma, oracle, sample = box
    fields = forward._fields(sigma)
    J = forward._jacobian_device(fields, False, None)
    assert J.shape == (4000, 244800)
    ours = J[torch.as_tensor(sample, device=J.device)].cpu().numpy()
    expected = oracle.jacobian(sigma.numpy().astype(float))
    for row in range(len(sample)):
        assert_close(ours[row], expected[row], 1e-4, f"3D box Jacobian row {sample[row]}")
    # a contiguous row range (rows in their own order) equals the same rows of the full launch
    part = torch.empty((100, forward.C), device=J.device)
    forward._call("adt_normal_jacobian", _native.ptr(fields), 1900, 100, _native.ptr(part), forward._stream())
    assert torch.equal(part, J[1900:2000])
