"""The reference's own GPU kernel against this library's Jacobian on the same fields.

``normal_sensitivity<float, 3>`` (adtlert/forward/kernels.py:132-178) is built by nvcc for
sm_100 from the reference's source into ``oracle/_ref`` (``oracle/reference_kernel.py``); this
pins the Jacobian to the reference's GPU code itself, not only to its CPU einsum. Skipped when
that library was not built (it needs the reference tree at build time)."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, synthetic
from cases import case_inputs
from conftest import assert_close
from oracle import reference_kernel as refk
from oracle.ert2p5d import Oracle2p5D

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refk.available(), reason="oracle/_ref reference kernel not built")]


def _reference_jacobian(forward, sigma, chunk=None):
    fields = forward._fields(sigma).total
    phi, a, b, m, n, cells, templates = refk.operator_inputs(forward, fields)
    D, C = forward.D, forward.C
    chunk = chunk or D
    out = torch.empty((D, C), dtype=torch.float32, device=fields.device)
    for start in range(0, D, chunk):
        sl = slice(start, min(D, start + chunk))
        part = torch.empty((sl.stop - sl.start, C), dtype=torch.float32, device=fields.device)
        refk.normal_sensitivity(phi, a[sl], b[sl], m[sl], n[sl], cells, templates, part)
        out[sl] = part
    torch.cuda.synchronize()
    return out.cpu()


def test_reference_kernel_matches_ours_and_the_oracle():
    inputs = case_inputs("tri_flat")
    forward = ERTForward2p5D(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                             Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    reference = _reference_jacobian(forward, sigma)
    assert_close(forward.jacobian(sigma), reference, 1e-4, "ours vs the reference kernel")
    oracle = Oracle2p5D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])
    assert_close(reference, oracle.normal_jacobian(inputs["sigma"]), 1e-4, "reference kernel vs FP64 oracle")
    # the reference launches 64 rows at a time; chunking changes no entry
    assert torch.equal(_reference_jacobian(forward, sigma, chunk=5), reference)


def test_reference_kernel_on_the_benchmark_section():
    nodes, cells, electrodes, rows = synthetic.flat_section()
    forward = ERTForward2p5D(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 3), dtype=torch.float32)
    reference = _reference_jacobian(forward, sigma, chunk=64)
    ours = forward.jacobian(sigma)
    assert np.isfinite(reference.numpy()).all()
    assert_close(ours, reference, 1e-4, "ours vs the reference kernel (1232 x 9600)")
