"""CUDA conductivities through the autograd bridge stay on the GPU.

A series on the GPU goes forward (resistances), backward (the exact VJP reusing the forward
factorization) and forward-mode (tangents) through the operator's device-resident entry points;
the field cache keys it with device fingerprints (16 bytes per model read back). Results equal
those of the CPU path, which is the reference's."""

import numpy as np
import pytest
import torch
import torch.autograd.forward_ad as fwAD

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, apparent_resistivity_autograd
from adtlert_b200 import _native
from adtlert_b200.field_store import model_fingerprints
from cases import case_inputs
from conftest import assert_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def forward():
    inputs = case_inputs("tri_flat")
    op = ERTForward2p5D(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                        Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    return op, inputs


def test_device_fingerprints_equal_host_fingerprints(forward):
    op, _ = forward
    rng = np.random.default_rng(1)
    for shape, dtype in (((5, 9600), torch.float32), ((3, 1001), torch.float64), ((1, 7), torch.float32)):
        models = torch.as_tensor(rng.uniform(0.01, 1.0, shape), dtype=dtype)
        host = model_fingerprints(op._lib, op._plan, models, op._stream())
        device = model_fingerprints(op._lib, op._plan, models.cuda(), op._stream())
        assert host == device


def test_cuda_series_goes_forward_and_backward_on_the_device(forward, monkeypatch):
    op, inputs = forward
    rng = np.random.default_rng(2)
    base = np.asarray(inputs["sigma"], dtype=np.float32)
    series = np.stack([base * rng.uniform(0.8, 1.25, base.shape).astype(np.float32) for _ in range(3)])
    weights = torch.as_tensor(rng.standard_normal((3, op.D)), dtype=torch.float32)

    cpu = torch.as_tensor(series).requires_grad_(True)
    out_cpu = apparent_resistivity_autograd(cpu, op)
    (out_cpu * weights).sum().backward()

    large = []
    real_cpu, real_numpy = torch.Tensor.cpu, torch.Tensor.numpy

    def watched_cpu(self, *a, **k):
        large.append(self.numel())
        return real_cpu(self, *a, **k)

    def watched_numpy(self, *a, **k):
        large.append(self.numel())
        return real_numpy(self, *a, **k)

    def refuse(*_a, **_k):
        raise AssertionError("a CUDA conductivity took the operator's CPU method")

    for name in ("resistance_series", "vjp_series", "jvp"):
        monkeypatch.setattr(ERTForward2p5D, name, refuse)
    monkeypatch.setattr(torch.Tensor, "cpu", watched_cpu)
    monkeypatch.setattr(torch.Tensor, "numpy", watched_numpy)
    gpu = torch.as_tensor(series, device="cuda").requires_grad_(True)
    launches = op.kernel_launches()
    out_gpu = apparent_resistivity_autograd(gpu, op)
    (out_gpu * weights.cuda()).sum().backward()
    torch.cuda.synchronize()
    monkeypatch.undo()
    assert op.kernel_launches() > launches
    assert out_gpu.device.type == "cuda" and gpu.grad.device.type == "cuda"
    assert max(large, default=0) < op.C, f"a host copy of {max(large)} elements was made"
    assert_close(out_gpu.detach().cpu(), out_cpu.detach(), 1e-6, "apparent resistivity, GPU vs CPU path")
    assert_close(gpu.grad.cpu(), cpu.grad, 1e-5, "conductivity gradient, GPU vs CPU path")


def test_forward_mode_on_the_device(forward):
    op, inputs = forward
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    direction = torch.as_tensor(np.random.default_rng(3).standard_normal(op.C), dtype=torch.float32) * sigma * 1e-2
    tangents = []
    for device in ("cpu", "cuda"):
        with fwAD.dual_level():
            dual = fwAD.make_dual(sigma.to(device), direction.to(device))
            _, tangent = fwAD.unpack_dual(apparent_resistivity_autograd(dual, op))
            assert tangent.device.type == device
            tangents.append(tangent.cpu())
    assert_close(tangents[1], tangents[0], 1e-5, "forward-mode tangent, GPU vs CPU path")
