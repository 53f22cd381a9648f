"""The surrogate's BF16 tensor-core kernels against float32/float64 references, and what the
trained network gains in the time-lapse inversion.

* adt_mlp_gemm (tcgen05, split-K) against torch's float32 matmul of the same BF16 operands
  (1e-5, max-norm relative), for the layer shapes of training and inference; bitwise repeatable.
* The backward pass (every weight and bias gradient of a 6144-1024-1024-1024-1280 network on a
  256 batch) against the float64 oracle given the same BF16-rounded weights and inputs: within
  1e-2 (BF16 activations and gradients between layers).
* Training on FEM data lowers the loss, and in the windowed inversion the screened run needs
  fewer FEM linearizations than the plain run at the same final misfit.
"""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, _native, synthetic
from adtlert_b200.surrogate import MLP, Surrogate, SurrogateScreen, training_set
from adtlert_b200.timelapse import WindowedInversion, WindowSettings
from conftest import assert_close
from oracle import surrogate as oracle

pytestmark = pytest.mark.gpu


def _bf16(rng, shape, scale=1.0):
    return torch.as_tensor(rng.standard_normal(shape) * scale, dtype=torch.float32, device="cuda").to(torch.bfloat16)


@pytest.mark.parametrize("m,n,k", [(256, 1024, 6144), (256, 1280, 1024), (128, 1024, 1024), (1280, 1024, 256),
                                   (1024, 6144, 256), (128, 128, 64)])
def test_gemm_matches_float32_matmul(m, n, k):
    rng = np.random.default_rng(m + n + k)
    net = MLP(6144, 1232, batch=256)
    a, b = _bf16(rng, (m, k)), _bf16(rng, (n, k))
    partial, splits = net.gemm(a, b, "test")
    out = torch.empty((m, n), dtype=torch.float32, device="cuda")
    net.epilogue(3, partial, splits, m, n, f32_out=out)
    again = torch.empty_like(out)
    partial, splits = net.gemm(a, b, "test")
    net.epilogue(3, partial, splits, m, n, f32_out=again)
    torch.cuda.synchronize()
    net.check_error()
    expected = a.float() @ b.float().T
    assert_close(out.cpu(), expected.cpu(), 1e-5, f"gemm {m}x{n}x{k} ({splits} splits)")
    assert torch.equal(out, again), "bitwise repeatable"


def test_backward_pass_matches_the_float64_oracle():
    rng = np.random.default_rng(7)
    net = MLP(6144, 1232, batch=256, seed=3)
    for layer in range(4):  # nonzero biases, so every term of the epilogues is exercised
        net.b[layer].copy_(torch.as_tensor(rng.standard_normal(net.b[layer].shape[0]) * 0.1))
    x16 = _bf16(rng, (256, 6144))
    xt16 = x16.T.contiguous()
    target = torch.as_tensor(rng.standard_normal((256, net.padded)), dtype=torch.float32, device="cuda")
    sums, dws, dbs = net.gradients(x16, xt16, target)
    torch.cuda.synchronize()
    net.check_error()
    weights = [w.float().cpu().numpy() for w in net.w16]
    biases = [b.cpu().numpy() for b in net.b]
    loss, ref_dw, ref_db = oracle.gradients(x16.float().cpu().numpy(), target.cpu().numpy(), weights, biases, 1232)
    assert abs(float(sums.sum()) / (256 * 1232) - loss) / loss < 1e-2
    for layer in range(4):
        assert_close(dws[layer].cpu(), ref_dw[layer], 1e-2, f"dW{layer + 1}")
        assert_close(dbs[layer].cpu(), ref_db[layer], 1e-2, f"db{layer + 1}")


def test_training_and_screening_gain():
    nodes, cells, electrodes, rows = synthetic.flat_section()
    forward = ERTForward2p5D(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    models, data = training_set(forward, 2048, seed=5)
    surrogate = Surrogate(forward, seed=1)
    history = surrogate.fit(models, data, epochs=8)
    assert history[-1] < 0.5 * history[0]
    # a short series: 6 steps of the infiltration workload, 4 windows
    rho = synthetic.infiltration_series(nodes, cells, 40, seed=0)[20:26]
    clean = forward.apparent_resistivity_series(torch.as_tensor(1.0 / rho, dtype=torch.float32)).numpy()
    observed = np.log(clean * np.exp(0.02 * np.random.default_rng(2).standard_normal(clean.shape)))
    initial = np.tile(np.median(observed, axis=1)[:, None], (1, len(cells)))
    settings = WindowSettings(data_std=float(np.log1p(0.02)))
    plain = WindowedInversion(forward, settings)
    plain_result = plain.run(observed, initial)
    screened = WindowedInversion(forward, settings)
    screen = SurrogateScreen(surrogate)
    screened_result = screened.run(observed, initial, screen=screen)
    plain_chi2 = [w["final_chi2"] for w in plain_result.windows]
    screened_chi2 = [w["final_chi2"] for w in screened_result.windows]
    assert max(screened_chi2) < 1.1 * max(plain_chi2)
    assert screened.linearize.evaluations < plain.linearize.evaluations, (screen.counts,
                                                                          screened.linearize.evaluations,
                                                                          plain.linearize.evaluations)
