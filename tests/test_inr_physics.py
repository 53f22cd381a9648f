"""The INR consumer of the operator: a coordinate network trained through
``matrix_free_log_rhoa_series`` (adtlert/inr/physics.py:70-89, as adtlert/inr/train.py:516-709
calls it each iteration).

A small network maps (cell centroid, time) to log-resistivity; its series of models goes forward
and backward through the operator's exact VJP on the GPU. The log apparent resistivities and the
gradient with respect to the network's log-resistivities are checked against the FP64 oracle
(-sigma times the oracle's exact VJP of the resistance with cotangent g / R), and a few Adam
steps must lower the misfit. Argument errors are checked on the CPU.
"""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey
from adtlert_b200 import inr
from cases import case_inputs
from conftest import assert_close


class _Facade:
    """An inversion facade exposing its operator, as the reference's forward-modeling wrappers do."""

    def __init__(self, operator):
        self.forward_operator = operator


def test_argument_errors_match_the_reference():
    with pytest.raises(TypeError, match="requires an ADTLERT ERTForward2p5D or ERTForward3D operator"):
        inr.forward_operator(object())
    with pytest.raises(ValueError, match="INR inversion runs on CUDA devices"):
        inr.select_cuda_device("cpu")
    with pytest.raises(TypeError, match="INR physics requires ERTForward2p5D"):
        inr._conductivity(object(), torch.zeros(3))


class _Network(torch.nn.Module):
    """Fourier-feature MLP of (x, z, t) -> log-resistivity (the shape of a coordinate network)."""

    def __init__(self, seed: int):
        super().__init__()
        generator = torch.Generator().manual_seed(seed)
        self.register_buffer("frequencies", torch.randn(3, 16, generator=generator) * 0.5)
        self.body = torch.nn.Sequential(torch.nn.Linear(32, 64), torch.nn.Tanh(), torch.nn.Linear(64, 1))
        with torch.no_grad():
            for layer in self.body:
                if isinstance(layer, torch.nn.Linear):
                    layer.weight.copy_(torch.randn(layer.weight.shape, generator=generator) * 0.2)
                    layer.bias.zero_()
        self.offset = torch.nn.Parameter(torch.tensor(np.log(50.0), dtype=torch.float32))

    def forward(self, coordinates):
        projected = coordinates @ self.frequencies
        return self.offset + self.body(torch.cat((torch.sin(projected), torch.cos(projected)), -1))[..., 0]


def _coordinates(inputs, steps, device):
    centers = inputs["nodes"][inputs["cells"]].mean(axis=1)
    span = np.abs(centers).max(axis=0)
    grid = []
    for t in range(steps):
        time = np.full((centers.shape[0], 1), t / max(steps - 1, 1))
        grid.append(np.hstack((centers / span, time)))
    return torch.as_tensor(np.stack(grid), dtype=torch.float32, device=device)


@pytest.mark.gpu
def test_coordinate_network_trains_through_the_exact_vjp():
    from oracle.ert2p5d import Oracle2p5D

    inputs = case_inputs("tri_flat")
    steps = 4
    operator = ERTForward2p5D(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                              Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    facade = _Facade(operator)
    report = inr.prepare_cuda_forward(facade, -np.log(inputs["sigma"]), device="cuda")
    assert report["gpu_device_index"] == torch.cuda.current_device()
    oracle = Oracle2p5D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])

    rng = np.random.default_rng(11)
    truth = np.stack([np.log(1.0 / inputs["sigma"]) + 0.3 * np.sin(0.7 * t + rng.uniform(0, 1, operator.C))
                      for t in range(steps)])
    observed = torch.as_tensor(np.stack([np.log(oracle.apparent_resistivity(np.exp(-m))) for m in truth]),
                               dtype=torch.float32, device="cuda")
    std = 0.02

    network = _Network(seed=5).cuda()
    coordinates = _coordinates(inputs, steps, "cuda")

    # one iteration: predictions and the model gradient against the oracle
    log_model = network(coordinates)
    log_model.retain_grad()
    prediction = inr.matrix_free_log_rhoa_series(log_model, facade)
    assert prediction.device.type == "cuda" and prediction.dtype == torch.float32
    misfit = 0.5 * (((prediction - observed) / std) ** 2).sum()
    misfit.backward()

    model = log_model.detach().double().cpu().numpy()
    residual = ((prediction.detach().double().cpu().numpy() - observed.double().cpu().numpy()) / std ** 2)
    for s in range(steps):
        sigma = np.exp(-model[s])
        expected = np.log(oracle.apparent_resistivity(sigma))
        assert_close(prediction[s].detach().cpu(), expected, 1e-4, f"log apparent resistivity, step {s}")
        # d misfit / d log rho = -sigma * d misfit / d sigma; d log rhoa / d R = 1 / R
        gradient = -sigma * oracle.vjp(sigma, residual[s] / oracle.resistance(sigma))
        assert_close(log_model.grad[s].cpu(), gradient, 5e-4, f"log-resistivity gradient, step {s}")

    single = inr.matrix_free_log_rhoa(log_model[1].detach(), operator)
    assert_close(single.cpu(), prediction[1].detach().cpu(), 1e-6, "one model against the series")

    # a few Adam steps through the operator lower the misfit
    optimizer = torch.optim.Adam(network.parameters(), lr=0.01)
    history = []
    for _ in range(8):
        optimizer.zero_grad()
        prediction = inr.matrix_free_log_rhoa_series(network(coordinates), facade)
        misfit = 0.5 * (((prediction - observed) / std) ** 2).sum()
        misfit.backward()
        optimizer.step()
        history.append(float(misfit))
    assert np.all(np.isfinite(history))
    assert history[-1] < history[0], f"misfit did not fall: {history}"
