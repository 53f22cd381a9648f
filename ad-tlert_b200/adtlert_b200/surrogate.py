"""Learned apparent-resistivity surrogate on hand-written BF16 tensor-core kernels.

A multilayer perceptron maps a section's log10 resistivity, sampled on a regular grid (128 x 48
over the flat section), to the survey's log10 apparent resistivities. Four layers, 1024 hidden
units, GELU (tanh form); BF16 weights and activations, FP32 accumulation, FP32 master weights
trained by Adam. Every GEMM is ``adt_mlp_gemm`` (tcgen05, TMEM accumulators); the epilogues
(bias, GELU and its derivative, transposed copies for the backward GEMMs), the loss, bias
gradients, Adam and the weight transposes are kernels of the same library. Training data come
from this library's FEM forward.

The reference has no surrogate (its inversion evaluates every candidate with the FEM). Here the
surrogate screens the line-search candidates of the windowed Gauss-Newton inversion
(``SurrogateScreen``): the step length is chosen on the surrogate's predicted change of the data,
only the accepted model is solved by the FEM, and whenever that FEM solve does not confirm a
lower objective the iteration falls back to the plain FEM candidate search.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .geometry import locate_points

Tensor = torch.Tensor
GRID = (128, 48)  # (x, depth) samples of the network input


def grid_cells(nodes: np.ndarray, cells: np.ndarray, shape=GRID) -> np.ndarray:
    """Index of the cell holding each point of a regular grid of cell-centred samples over the
    section's bounding box (row-major: depth outer, x inner)."""

    nx, nz = shape
    xmin, zmin = nodes.min(axis=0)
    xmax, zmax = nodes.max(axis=0)
    xs = xmin + (np.arange(nx) + 0.5) * (xmax - xmin) / nx
    zs = zmax - (np.arange(nz) + 0.5) * (zmax - zmin) / nz
    points = np.column_stack([np.tile(xs, nz), np.repeat(zs, nx)])
    ids, _ = locate_points(nodes, cells, points)
    if np.any(ids < 0):
        raise ValueError("grid points outside the mesh")
    return ids.astype(np.int64)


def _pad(value: int, multiple: int) -> int:
    return -(-value // multiple) * multiple


class MLP:
    """The network and its training state (all on one GPU)."""

    def __init__(self, inputs: int, outputs: int, hidden: int = 1024, layers: int = 4, batch: int = 256,
                 seed: int = 0, device=None) -> None:
        if inputs % 64 or hidden % 128 or batch % 128:
            raise ValueError("inputs must be a multiple of 64, hidden and batch multiples of 128")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.lib = _native.load_library()
        self.inputs, self.outputs, self.hidden, self.batch = inputs, outputs, hidden, batch
        self.padded = _pad(outputs, 128)
        self.sizes = [inputs] + [hidden] * (layers - 1) + [self.padded]
        self.multiprocessors = torch.cuda.get_device_properties(self.device).multi_processor_count
        rng = np.random.default_rng(seed)
        dev = self.device
        self.w, self.b, self.w16, self.wt16 = [], [], [], []
        for layer in range(layers):
            fan_in, fan_out = self.sizes[layer], self.sizes[layer + 1]
            w = rng.standard_normal((fan_out, fan_in)) * math.sqrt(2.0 / fan_in)
            if layer == layers - 1:
                w[outputs:] = 0.0
                w *= 0.5
            self.w.append(torch.as_tensor(w, dtype=torch.float32, device=dev).contiguous())
            self.b.append(torch.zeros(fan_out, dtype=torch.float32, device=dev))
            self.w16.append(torch.empty((fan_out, fan_in), dtype=torch.bfloat16, device=dev))
            self.wt16.append(torch.empty((fan_in, fan_out), dtype=torch.bfloat16, device=dev) if layer > 0 else None)
        self.moments = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.w + self.b]
        self.steps = 0
        self.error = torch.zeros(1, dtype=torch.int32, device=dev)
        self.launches = 0
        self._buffers = {}
        self._refresh_bf16()

    # ---------------------------------------------------------------- kernels
    def _stream(self):
        return _native.stream_handle(self.device)

    def _check(self, status: int, what: str) -> None:
        self.launches += 1
        if status != _native.ADT_OK:
            raise RuntimeError(f"{what} failed with status {status}")

    def _buffer(self, name: str, shape, dtype) -> Tensor:
        key = (name, tuple(shape), dtype)
        if key not in self._buffers:
            self._buffers[key] = torch.empty(shape, dtype=dtype, device=self.device)
        return self._buffers[key]

    def _refresh_bf16(self) -> None:
        for layer, w in enumerate(self.w):
            self._check(self.lib.adt_mlp_to_bf16(_native.ptr(w), w.numel(), _native.ptr(self.w16[layer]), self._stream()),
                        "adt_mlp_to_bf16")
            if self.wt16[layer] is not None:
                rows, cols = w.shape
                self._check(self.lib.adt_mlp_transpose(_native.ptr(self.w16[layer]), rows, cols,
                                                       _native.ptr(self.wt16[layer]), self._stream()),
                            "adt_mlp_transpose")

    def gemm(self, a: Tensor, b: Tensor, tag: str) -> tuple[Tensor, int]:
        """FP32 split partials of a b^T (a: m x k, b: n x k, BF16) and the split count."""

        m, k = a.shape
        n = b.shape[0]
        splits = int(self.lib.adt_mlp_gemm_splits(m, n, k, self.multiprocessors))
        partial = self._buffer(f"partial:{tag}", (splits, m, n), torch.float32)
        self._check(self.lib.adt_mlp_gemm(_native.ptr(a), _native.ptr(b), m, n, k, splits, _native.ptr(partial),
                                          partial.numel(), _native.ptr(self.error), self._stream()), "adt_mlp_gemm")
        return partial, splits

    def epilogue(self, mode: int, partial: Tensor, splits: int, m: int, n: int, *, bias=None, z_in=None, z_out=None,
                 row_out=None, col_out=None, f32_out=None) -> None:
        p = _native.ptr
        self._check(self.lib.adt_mlp_epilogue(mode, p(partial), splits, m, n, p(bias), p(z_in), p(z_out), p(row_out),
                                              p(col_out), p(f32_out), self._stream()), "adt_mlp_epilogue")

    # ---------------------------------------------------------------- passes
    def forward(self, x16: Tensor, keep: bool = False) -> Tensor:
        """FP32 outputs (M, padded) of BF16 inputs (M, inputs); ``keep`` stores the pre-activations
        and transposed activations the backward pass reads."""

        m = int(x16.shape[0])
        act, last = x16, len(self.w) - 1
        for layer in range(last):
            n = self.sizes[layer + 1]
            partial, splits = self.gemm(act, self.w16[layer], "forward")
            z = self._buffer(f"z{layer}", (m, n), torch.bfloat16)
            y = self._buffer(f"y{layer}", (m, n), torch.bfloat16)
            yt = self._buffer(f"yt{layer}", (n, m), torch.bfloat16) if keep else None
            self.epilogue(0, partial, splits, m, n, bias=self.b[layer], z_out=z, row_out=y, col_out=yt)
            act = y
        out = self._buffer("out", (m, self.padded), torch.float32)
        partial, splits = self.gemm(act, self.w16[last], "forward")
        self.epilogue(1, partial, splits, m, self.padded, bias=self.b[last], f32_out=out)
        return out

    def gradients(self, x16: Tensor, xt16: Tensor, target: Tensor):
        """Loss sums (device) and the FP32 gradients (dW, db per layer) of the mean squared error
        of a batch: the network's backward pass, every GEMM on the tensor cores."""

        m, last = int(x16.shape[0]), len(self.w) - 1
        out = self.forward(x16, keep=True)
        g = self._buffer("g_out", (m, self.padded), torch.bfloat16)
        gt = self._buffer("gt_out", (self.padded, m), torch.bfloat16)
        sums = self._buffer("loss_sums", ((m // 32) * (self.padded // 32),), torch.float32)
        self._check(self.lib.adt_mlp_loss(_native.ptr(out), _native.ptr(target), m, self.padded, self.outputs,
                                          _native.ptr(g), _native.ptr(gt), _native.ptr(sums), self._stream()),
                    "adt_mlp_loss")
        dws, dbs = [None] * (last + 1), [None] * (last + 1)
        for layer in range(last, -1, -1):
            n_out, n_in = self.sizes[layer + 1], self.sizes[layer]
            previous = xt16 if layer == 0 else self._buffer(f"yt{layer - 1}", (n_in, m), torch.bfloat16)
            partial, splits = self.gemm(gt, previous, "backward")
            dws[layer] = self._buffer(f"dw{layer}", (n_out, n_in), torch.float32)
            self.epilogue(3, partial, splits, n_out, n_in, f32_out=dws[layer])
            dbs[layer] = self._buffer(f"db{layer}", (n_out,), torch.float32)
            self._check(self.lib.adt_mlp_bias_grad(_native.ptr(gt), n_out, m, _native.ptr(dbs[layer]), self._stream()),
                        "adt_mlp_bias_grad")
            if layer > 0:
                partial, splits = self.gemm(g, self.wt16[layer], "backward")
                g_prev = self._buffer(f"g{layer - 1}", (m, n_in), torch.bfloat16)
                gt_prev = self._buffer(f"gt{layer - 1}", (n_in, m), torch.bfloat16)
                z = self._buffer(f"z{layer - 1}", (m, n_in), torch.bfloat16)
                self.epilogue(2, partial, splits, m, n_in, z_in=z, row_out=g_prev, col_out=gt_prev)
                g, gt = g_prev, gt_prev
        return sums, dws, dbs

    def train_step(self, x16: Tensor, xt16: Tensor, target: Tensor, lr: float = 1e-3, beta1: float = 0.9,
                   beta2: float = 0.999, eps: float = 1e-8) -> Tensor:
        """One Adam step on a batch; returns the device sums of the batch's squared errors."""

        sums, dws, dbs = self.gradients(x16, xt16, target)
        self.steps += 1
        c1, c2 = 1.0 / (1.0 - beta1 ** self.steps), 1.0 / (1.0 - beta2 ** self.steps)
        params = self.w + self.b
        grads = dws + dbs
        copies = self.w16 + [None] * len(self.b)
        for param, grad, (first, second), copy in zip(params, grads, self.moments, copies, strict=True):
            self._check(self.lib.adt_mlp_adam(_native.ptr(param), _native.ptr(grad), _native.ptr(first),
                                              _native.ptr(second), param.numel(), lr, beta1, beta2, eps, c1, c2,
                                              _native.ptr(copy), self._stream()), "adt_mlp_adam")
        for layer in range(1, len(self.w)):
            rows, cols = self.w[layer].shape
            self._check(self.lib.adt_mlp_transpose(_native.ptr(self.w16[layer]), rows, cols,
                                                   _native.ptr(self.wt16[layer]), self._stream()), "adt_mlp_transpose")
        return sums

    def check_error(self) -> None:
        if int(self.error.item()) != 0:
            raise RuntimeError("a surrogate GEMM gave up waiting on its tensor-core pipeline (bounded wait ran out)")


class Surrogate:
    """log apparent resistivity of a flat-section operator's survey from log resistivity models."""

    def __init__(self, forward, *, hidden: int = 1024, layers: int = 4, batch: int = 256, seed: int = 0) -> None:
        self.forward_operator = forward
        self.device = forward.device
        mesh = forward.mesh
        self.cells = torch.as_tensor(grid_cells(mesh.nodes, mesh.cells), device=self.device)
        self.mlp = MLP(self.cells.numel(), forward.D, hidden=hidden, layers=layers, batch=batch, seed=seed,
                       device=self.device)
        self.x_shift, self.x_scale = 2.0, 1.0  # log10 resistivity standardization
        self.y_shift = torch.zeros(forward.D, dtype=torch.float64, device=self.device)
        self.y_scale = torch.ones(forward.D, dtype=torch.float64, device=self.device)
        self.history: list[float] = []

    # ---------------------------------------------------------------- data
    def _inputs(self, log10_models: Tensor, rows: int) -> Tensor:
        """BF16 network inputs (rows, 6144) of (n <= rows, C) log10 models; extra rows are zero."""

        x = torch.zeros((rows, self.cells.numel()), dtype=torch.float32, device=self.device)
        n = int(log10_models.shape[0])
        x[:n] = ((log10_models.to(self.device, torch.float32)[:, self.cells] - self.x_shift) / self.x_scale)
        x16 = torch.empty(x.shape, dtype=torch.bfloat16, device=self.device)
        self.mlp._check(self.mlp.lib.adt_mlp_to_bf16(_native.ptr(x), x.numel(), _native.ptr(x16), self.mlp._stream()),
                        "adt_mlp_to_bf16")
        return x16

    def _targets(self, log10_data: Tensor, rows: int) -> Tensor:
        y = torch.zeros((rows, self.mlp.padded), dtype=torch.float32, device=self.device)
        n = int(log10_data.shape[0])
        y[:n, :self.mlp.outputs] = ((log10_data.to(self.device, torch.float64) - self.y_shift) / self.y_scale).float()
        return y

    # ---------------------------------------------------------------- training
    def fit(self, log10_models, log10_data, *, epochs: int = 30, lr: float = 1e-3, final_lr: float = 5e-5,
            seed: int = 1) -> list[float]:
        """Adam on mini-batches of (S, C) log10 models and (S, D) log10 apparent resistivities
        (both on the GPU); the learning rate decays geometrically to ``final_lr``. Returns the
        mean squared error (standardized units) per epoch."""

        models = torch.as_tensor(log10_models, device=self.device)
        data = torch.as_tensor(log10_data, device=self.device, dtype=torch.float64)
        self.x_shift = float(models.float().mean())
        self.x_scale = float(models.float().std())
        self.y_shift = data.mean(dim=0)
        self.y_scale = data.std(dim=0).clamp(min=1e-6)
        count, batch = int(models.shape[0]), self.mlp.batch
        steps_per_epoch = count // batch
        total = max(1, epochs * steps_per_epoch)
        decay = (final_lr / lr) ** (1.0 / total)
        generator = torch.Generator(device="cpu").manual_seed(seed)
        step = 0
        for _ in range(epochs):
            order = torch.randperm(count, generator=generator).to(self.device)
            sums = []
            for start in range(0, steps_per_epoch * batch, batch):
                chosen = order[start:start + batch]
                x16 = self._inputs(models[chosen], batch)
                xt16 = torch.empty((x16.shape[1], batch), dtype=torch.bfloat16, device=self.device)
                self.mlp._check(self.mlp.lib.adt_mlp_transpose(_native.ptr(x16), batch, x16.shape[1], _native.ptr(xt16),
                                                               self.mlp._stream()), "adt_mlp_transpose")
                sums.append(self.mlp.train_step(x16, xt16, self._targets(data[chosen], batch), lr=lr * decay ** step)
                            .sum())
                step += 1
            self.history.append(float(torch.stack(sums).sum()) / (steps_per_epoch * batch * self.mlp.outputs))
        self.mlp.check_error()
        return self.history

    # ---------------------------------------------------------------- inference
    def predict_log10(self, log10_models: Tensor) -> Tensor:
        """(n, D) log10 apparent resistivities of (n, C) log10 models (float64, on the GPU)."""

        n = int(log10_models.shape[0])
        rows = _pad(max(n, 1), 128)
        out = self.mlp.forward(self._inputs(log10_models, rows))
        return out[:n, :self.mlp.outputs].double() * self.y_scale + self.y_shift

    def predict(self, log_models: Tensor) -> Tensor:
        """Natural-log apparent resistivities of natural-log resistivity models (n, C)."""

        return self.predict_log10(log_models / math.log(10.0)) * math.log(10.0)


def training_set(forward, count: int, seed: int = 0, batch: int = 8):
    """(count, C) log10 resistivity models and their (count, D) log10 apparent resistivities by
    this library's FEM forward. Models: the flat workload's seeded layered models with two
    Gaussian anomalies; three in four also carry an infiltration front (depth U(0, 8) m,
    resistivity above it times U(0.3, 0.7)) as the time-lapse series does."""

    from . import synthetic

    mesh = forward.mesh
    depth = -mesh.nodes[mesh.cells].mean(axis=1)[:, 1]
    rng = np.random.default_rng(seed + 104729)
    rho = np.empty((count, mesh.cell_count), dtype=np.float64)
    for i in range(count):
        base = 1.0 / synthetic.layered_model(mesh.nodes, mesh.cells, seed * 1_000_003 + i).astype(float)
        if rng.uniform() < 0.75:
            front, factor = rng.uniform(0.0, 8.0), rng.uniform(0.3, 0.7)
            base = np.where(depth < front, base * factor, base)
        rho[i] = base
    data = []
    sigma = torch.as_tensor(1.0 / rho, dtype=torch.float32, device=forward.device)
    factors = forward._geometric_factors().to(forward.device, torch.float64)
    for start in range(0, count, batch):
        resistance = forward._resistances_device(sigma[start:start + batch]).double()
        data.append(torch.log10(factors * resistance))
    return torch.as_tensor(np.log10(rho), device=forward.device), torch.cat(data)


class SurrogateScreen:
    """Candidate screening of the windowed Gauss-Newton inversion.

    Window candidates (on by default): a window may start from the reference's initial models or
    from the preceding window's result moved one step on (its last model repeated; those models
    are in the linearization cache, so that start costs no FEM solve). The surrogate estimates the
    objective of both and only the one chosen is linearized by the FEM; when the FEM objective of
    a warm start exceeds the surrogate's estimate for the reference's start, the window falls back
    to the reference's start. Windows started near their solution need fewer Gauss-Newton
    iterations (measured on 30 windows of the flat time-lapse workload: 5.0 -> 2.2 iterations,
    630 -> 201 FEM model solves, 2.8x faster, mean final chi2 1.052 -> 1.048).

    Line-search candidates (``line_search=True``, off by default): the reference solves the FEM at
    the full-step candidate and, when the grid search along the step picks tau < 0.95, again at
    the chosen model (adtlert/inversion/core.py:224-257, objective.py:168-192). Screened, the search
    runs on the FEM data at the current model plus the surrogate's predicted change of the data,
    the FEM solves only the chosen model and falls back to the FEM search when the objective there
    is not lower. A surrogate accurate to a few percent in absolute apparent resistivity is far
    less accurate in the small change along one step, so the screened search picked shorter
    steps and the windows needed more iterations (measured: 5.0 -> 14.5 iterations); it is kept
    as an option.

    With ``surrogate=None`` the window candidates are judged by the FEM itself (the reference's
    start linearized too), the variant that shows what the network adds to the warm start.

    A warm-started window also stops when an iteration changes its data chi2 by at most
    ``stall_tolerance`` (relative): started next to a solution, some windows otherwise keep
    taking full steps along a direction that changes neither the data nor the objective until the
    iteration limit (measured on the 363-window run: 67 windows at 15 iterations with chi2
    constant to 1e-4). It also stops after its second or later step when the line search's
    quadratic predicts that step lowered the objective by less than ``objective_tolerance``
    (relative): from a warm start the first step lowers the objective by ~3 %, the second by
    0.01-0.2 %, later ones by less than 1e-4 (measured on the same run), so 3e-3 ends most warm
    windows after their second step. Its Gauss-Newton steps run at most ``cgls_iterations`` CGLS
    iterations instead of the settings' count: a step from next to the solution needs no fully
    converged inner solve. Measured on the same run, the final chi2 and the ρa error stayed
    within 0.6 % of the plain run's for every pair swept (objective tolerance 1e-3, 3e-3, 1e-2;
    CGLS 60 down to 10), and (3e-3, 20) gave the most windows per second among the pairs that
    kept about two iterations per window. The windows started from the reference's models keep
    the reference's stop rules and CGLS count.
    """

    def __init__(self, surrogate: Surrogate | None, *, warm_start: bool = True, line_search: bool = False,
                 stall_tolerance: float | None = 1.0e-4, objective_tolerance: float | None = 3.0e-3,
                 cgls_iterations: int | None = 20) -> None:
        self.surrogate = surrogate
        self.warm_start = warm_start
        self.line_search = line_search
        self.stall_tolerance = stall_tolerance
        self.objective_tolerance = objective_tolerance
        self.cgls_iterations = cgls_iterations
        self.counts = {"line_search_screened": 0, "line_search_fallbacks": 0, "warm_starts": 0,
                       "warm_start_fallbacks": 0, "surrogate_batches": 0, "stalled_windows": 0,
                       "converged_windows": 0}

    def _objectives(self, inv, candidates: Tensor, observed: Tensor, weights: Tensor, steps: int) -> list[float]:
        if self.surrogate is None:
            predicted = torch.cat([inv.linearize(candidates[i:i + steps])[0]
                                   for i in range(0, int(candidates.shape[0]), steps)])
        else:
            predicted = self.surrogate.predict(candidates)
            self.counts["surrogate_batches"] += 1
        values = []
        for i in range(0, int(candidates.shape[0]), steps):
            values.append(inv.objective(candidates[i:i + steps], predicted[i:i + steps], observed, weights))
        return torch.stack(values).cpu().tolist()

    def screened_step(self, inv, models, step, candidate, predicted, observed, weights, result):
        from .timelapse import line_search_tau

        if not self.line_search or self.surrogate is None:
            return None
        steps = int(models.shape[0])
        surrogate = self.surrogate.predict(torch.cat([models, candidate]))
        self.counts["surrogate_batches"] += 1
        change = surrogate[steps:] - surrogate[:steps]
        residual0 = weights * (predicted - observed)
        tau = line_search_tau(inv.quadratic(models, step, residual0, weights * change))
        if tau <= 0.0:
            return None  # no descent predicted: the FEM search decides
        chosen = candidate if tau >= 0.95 else inv._clip(models + tau * step).contiguous()
        chosen_predicted, chosen_J = inv.linearize(chosen)
        before = inv.objective(models, predicted, observed, weights)
        after = inv.objective(chosen, chosen_predicted, observed, weights)
        if float(after) < float(before):
            result.screened += 1
            self.counts["line_search_screened"] += 1
            return tau, tau * step, chosen, chosen_predicted, chosen_J
        result.fallbacks += 1
        self.counts["line_search_fallbacks"] += 1
        return None

    def window_start(self, inv, observed: Tensor, initial: Tensor, previous: Tensor | None):
        """(start models, objective bound or None): the reference's initial models, or the
        previous window's models one step on when the surrogate rates them lower."""

        if not self.warm_start or previous is None:
            return initial, None
        steps = int(initial.shape[0])
        warm = torch.cat([previous[1:], previous[-1:]]).contiguous()
        weights = torch.full((steps, inv.forward.D), 1.0 / float(inv.settings.data_std), dtype=torch.float64,
                             device=inv.device)
        reference_estimate, warm_estimate = self._objectives(inv, torch.cat([inv._clip(initial), warm]), observed,
                                                             weights, steps)
        if warm_estimate >= reference_estimate:
            return initial, None
        self.counts["warm_starts"] += 1
        return warm, reference_estimate

    def reject_start(self) -> None:
        self.counts["warm_start_fallbacks"] += 1
