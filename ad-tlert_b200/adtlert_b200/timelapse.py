"""Windowed time-lapse Gauss-Newton inversion with every step on the GPU.

The caller of the forward path in AD-TLERT's time-lapse workflow is its sliding-window
inversion (adtlert/inversion/core.py:445-577 -> _invert, core.py:81-300). This module runs the
same algorithm for the configuration the reference's 363-window example uses
(example/window_363/inversion_adtlert.py:483-603): log-resistivity state, weighted log L2 data
misfit, first-order spatial smoothness and first-order temporal smoothness in the "model" mode,
Gauss-Newton steps solved by CGLS, a grid line search along the step, model bounds, and windows
inverted independently from the initial models, each time step's result the mean of the log
models of the windows that contain it.

What changes is where it runs. The reference builds a SciPy CSR matrix from the dense host
Jacobians at every iteration and ships it to the GPU for CGLS. Here the Jacobians are formed on
the GPU by the library (fields, sensitivity kernel, log chain rule applied on the device) and
stay there; the CGLS step (adt_gn_step) reads them in place with the regularization applied
matrix-free, and the line search evaluates its objective as a quadratic in the step length
from a few device dot products. Per iteration the host reads back a handful of scalars.

A learned surrogate may screen candidate models (``screen=``): see ``surrogate.py``.
"""

from __future__ import annotations

import ctypes
import math
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from .ert2p5d import ERTForward2p5D
from .field_store import model_fingerprints

Tensor = torch.Tensor


@dataclass(frozen=True)
class WindowSettings:
    """Settings of the windowed inversion (names as in adtlert/inversion/config.py:33-96; the
    defaults are the 363-window example's, example/window_363/inversion_adtlert.py:483-603)."""

    max_iterations: int = 15
    data_std: float = 0.05
    regularization: float = 50.0
    temporal_regularization: float = 10.0
    z_weight: float = 1.0
    model_bounds: tuple[float, float] | None = (0.001, 1.0e4)
    step_length: float = 1.0
    max_log_step: float | None = None
    line_search: bool = True
    step_tolerance: float = 1.0e-4
    target_chi2: float | None = None
    cgls_max_iterations: int = 60
    cgls_tolerance: float = 1.0e-12

    def log_bounds(self):
        if self.model_bounds is None:
            return None
        low, high = self.model_bounds
        return math.log(low), math.log(high)


def neighbour_graph(nodes: np.ndarray, cells: np.ndarray, z_weight: float = 1.0):
    """Symmetric neighbour lists of the first-order smoothness operator: cells sharing an edge,
    row weight 1 + |n_z| (z_weight - 1) of the shared edge's unit normal
    (adtlert/inversion/regularization.py:97-141). Returns (ptr, cells, squared weights)."""

    cells = np.asarray(cells, dtype=np.int64)
    count, k = cells.shape
    a = cells
    b = np.roll(cells, -1, axis=1)
    edges = np.sort(np.stack([a, b], axis=2).reshape(-1, 2), axis=1)
    owner = np.repeat(np.arange(count), k)
    order = np.lexsort((owner, edges[:, 1], edges[:, 0]))
    edges, owner = edges[order], owner[order]
    same = np.all(edges[1:] == edges[:-1], axis=1)
    first = np.flatnonzero(same)
    left, right = owner[first], owner[first + 1]
    tangent = np.asarray(nodes, dtype=float)[edges[first, 1]] - np.asarray(nodes, dtype=float)[edges[first, 0]]
    length = np.linalg.norm(tangent, axis=1)
    keep = length > 0.0
    left, right = left[keep], right[keep]
    normal_z = np.abs(tangent[keep, 0]) / length[keep]  # normal (-t_y, t_x): its z part is t_x
    weight2 = (1.0 + normal_z * (float(z_weight) - 1.0)) ** 2
    src = np.concatenate([left, right])
    dst = np.concatenate([right, left])
    w2 = np.concatenate([weight2, weight2])
    order = np.lexsort((dst, src))
    src, dst, w2 = src[order], dst[order], w2[order]
    ptr = np.zeros(count + 1, dtype=np.int32)
    np.add.at(ptr, src + 1, 1)
    return np.cumsum(ptr).astype(np.int32), dst.astype(np.int32), w2.astype(np.float64)


class Linearizer:
    """log apparent resistivities and d log(rhoa) / d log(rho) of model batches on the GPU
    (adtlert/forward/modeling.py:137-162 as the inversion calls it,
    adtlert/inversion/forward_calls.py:40-72), with an LRU of per-model results keyed by the
    model's content (the reference's linearization cache, forward_calls.py:57-72)."""

    def __init__(self, forward: ERTForward2p5D, capacity: int = 12, slot: int = 13) -> None:
        self.forward = forward
        self.device = forward.device
        self.capacity = int(capacity)
        self.slot = int(slot)
        self._recent: OrderedDict = OrderedDict()
        self._factors = forward._geometric_factors().to(self.device, torch.float32)
        self.evaluations = 0  # models solved (cache misses)
        self.requests = 0

    def _keys(self, log_models: Tensor) -> list[bytes]:
        f = self.forward
        return model_fingerprints(f._lib, f._plan, log_models, f._stream())

    def _solve(self, log_models: Tensor, jacobian: bool):
        f = self.forward
        T = int(log_models.shape[0])
        D, C, W, N, E = f.D, f.C, f.W, f.N, f.E
        sigma = torch.exp(-log_models).to(torch.float32).contiguous()
        fields = torch.empty((T, W, N, E), dtype=torch.float32, device=self.device)
        normal = torch.empty((T, D), dtype=torch.float64, device=self.device)
        reciprocal = torch.empty_like(normal)
        stream = f._stream()
        f._call("adt_factorize_fields", self.slot, _native.ptr(sigma), T, stream)
        f._call("adt_solve_fields", self.slot, _native.ptr(sigma), T, _native.ptr(fields), stream)
        f._call("adt_measure", _native.ptr(fields), T, _native.ptr(normal), _native.ptr(reciprocal), None, stream)
        resistance = (torch.sign(normal) * torch.sqrt(torch.abs(normal * reciprocal))).to(torch.float32)
        apparent = self._factors * resistance  # float32, as the operator's response
        predicted = torch.log(apparent.to(torch.float64))
        if not jacobian:
            return predicted, None
        J = torch.empty((T, D, C), dtype=torch.float32, device=self.device)
        row_scale = (self._factors[None] / apparent).to(torch.float64).contiguous()
        column_scale = (-sigma).to(torch.float64).contiguous()
        for t in range(T):
            f._call("adt_normal_jacobian", _native.ptr(fields[t]), 0, D, _native.ptr(J[t]), stream)
            _native.check(f._lib.adt_scale_rows_columns(_native.ptr(J[t]), D, C, _native.ptr(row_scale[t]),
                                                        _native.ptr(column_scale[t]), stream), f._plan,
                          "adt_scale_rows_columns")
        return predicted, J

    def _remember(self, keys, predicted, J) -> None:
        if self.capacity <= 0:
            return
        for t, key in enumerate(keys):
            self._recent[key] = (predicted[t], None if J is None else J[t])
            self._recent.move_to_end(key)
        while len(self._recent) > self.capacity:
            self._recent.popitem(last=False)

    def __call__(self, log_models: Tensor, jacobian: bool = True):
        """(T, D) predicted log data and, with ``jacobian``, the (T, D, C) log Jacobians."""

        T = int(log_models.shape[0])
        keys = self._keys(log_models)
        self.requests += T
        found = {}
        for t, key in enumerate(keys):
            hit = self._recent.get(key)
            if hit is not None and (hit[1] is not None or not jacobian):
                self._recent.move_to_end(key)
                found[t] = hit
        missing = [t for t in range(T) if t not in found]
        if len(missing) == T:  # nothing cached: the solved batch is returned as is (no copy)
            predicted, J = self._solve(log_models.contiguous(), jacobian)
            self.evaluations += T
            self._remember(keys, predicted, J)
            return predicted, J
        if missing:
            predicted, J = self._solve(log_models[missing].contiguous(), jacobian)
            self.evaluations += len(missing)
            for i, t in enumerate(missing):
                found[t] = (predicted[i], None if J is None else J[i])
                if self.capacity > 0:
                    self._recent[keys[t]] = found[t]
                    self._recent.move_to_end(keys[t])
            while len(self._recent) > self.capacity:
                self._recent.popitem(last=False)
        predicted = torch.stack([found[t][0] for t in range(T)])
        if not jacobian:
            return predicted, None
        return predicted, torch.stack([found[t][1] for t in range(T)])


def line_search_tau(quadratic: tuple[float, float, float], data_at_one: float | None = None) -> float:
    """Step length of the reference's grid line search (adtlert/inversion/objective.py:168-192).

    Along the step the objective is phi(tau) = a0 + 2 a1 tau + a2 tau^2: the data term is taken
    linear in tau between the current and the candidate predictions, and the regularization is
    quadratic. tau = 1 when phi(1) < phi(0); otherwise the best of tau = 0.01, ..., 1.00 that
    improves on phi(0), with 0 < tau < 0.03 raised to 0.03."""

    a0, a1, a2 = quadratic

    def phi(tau: float) -> float:
        return a0 + 2.0 * a1 * tau + a2 * tau * tau

    best_phi = phi(0.0)
    if phi(1.0) < best_phi:
        return 1.0
    best_tau = 0.0
    for index in range(1, 101):
        tau = 0.01 * index
        value = phi(tau)
        if value < best_phi:
            best_phi, best_tau = value, tau
    return 0.03 if 0.0 < best_tau < 0.03 else best_tau


@dataclass
class WindowResult:
    log_models: Tensor              # (T, C) final log resistivities
    predicted_log: Tensor           # (T, D) at the final models
    chi2: list[float]               # per iteration
    taus: list[float] = field(default_factory=list)
    stop_reason: str = "max_iterations"
    screened: int = 0               # candidates judged by the surrogate alone
    fallbacks: int = 0              # screened candidates the FEM rejected


class WindowedInversion:
    """Gauss-Newton inversion of time-lapse windows on one GPU (see the module docstring)."""

    def __init__(self, forward: ERTForward2p5D, settings: WindowSettings | None = None, *,
                 cache_models: int = 12) -> None:
        self.forward = forward
        self.settings = settings or WindowSettings()
        self.device = forward.device
        mesh = forward.mesh
        ptr, cells, w2 = neighbour_graph(mesh.nodes, mesh.cells, self.settings.z_weight)
        self._graph = tuple(torch.as_tensor(a, device=self.device) for a in (ptr, cells, w2))
        self.linearize = Linearizer(forward, capacity=cache_models)
        self._workspace = None
        self._workspace_key = None
        self.multiprocessors = torch.cuda.get_device_properties(self.device).multi_processor_count

    # ---------------------------------------------------------------- pieces
    def _clip(self, log_models: Tensor) -> Tensor:
        bounds = self.settings.log_bounds()
        return log_models if bounds is None else log_models.clamp(*bounds)

    def _ensure_workspace(self, T: int) -> None:
        f = self.forward
        key = (T, f.D, f.C)
        if self._workspace_key == key:
            return
        size = ctypes.c_size_t()
        _native.check(f._lib.adt_gn_workspace_bytes(T, f.D, f.C, self.multiprocessors, ctypes.byref(size)), f._plan,
                      "adt_gn_workspace_bytes")
        self._workspace = torch.empty(int(size.value) + 256, dtype=torch.uint8, device=self.device)
        self._workspace_key = key

    def _workspace_ptr(self):
        base = self._workspace.data_ptr()
        return (base + 255) & ~255, self._workspace.numel() - ((-base) % 256)

    def gauss_newton_step(self, J: Tensor, weights: Tensor, rhs: Tensor, models: Tensor,
                          iterations: int | None = None) -> Tensor:
        """CGLS solution (T, C) float64 of the linearized window system (adt_gn_step), with at most
        ``iterations`` CGLS iterations (default: the settings' ``cgls_max_iterations``)."""

        f, s = self.forward, self.settings
        T = int(models.shape[0])
        self._ensure_workspace(T)
        step = torch.empty((T, f.C), dtype=torch.float64, device=self.device)
        address, size = self._workspace_ptr()
        ptr, cells, w2 = self._graph
        _native.check(f._lib.adt_gn_step(
            f._plan, _native.ptr(J), T, f.D, f.C, _native.ptr(weights), _native.ptr(rhs), _native.ptr(models),
            _native.ptr(ptr), _native.ptr(cells), _native.ptr(w2), float(s.regularization),
            float(s.temporal_regularization), int(s.cgls_max_iterations if iterations is None else iterations),
            float(s.cgls_tolerance),
            _native.ptr(step), address, size, self.multiprocessors, f._stream()), f._plan, "adt_gn_step")
        return step

    def _cgls_state(self) -> Tensor:
        """The last step's device state as int32 words (the workspace's first 16 bytes: done,
        iterations, error, reserved; the float64 gammas follow)."""

        address, _ = self._workspace_ptr()
        offset = address - self._workspace.data_ptr()
        return self._workspace[offset:offset + 16].view(torch.int32)

    def cgls_iterations(self) -> int:
        """CGLS iterations the last ``gauss_newton_step`` ran before its stop test held. Synchronizes."""

        return int(self._cgls_state()[1].item())

    def _check_cgls(self, error: float) -> None:
        if error != 0:
            raise RuntimeError("adt_gn_step: a data pass gave up waiting for its copies of the Jacobian rows "
                               "(the step is NaN)")

    def regularized(self, models: Tensor) -> Tensor:
        """(ls R^T R + lt D^T D) models, (T, C) float64 on the device (adt_gn_regularize)."""

        f, s = self.forward, self.settings
        out = torch.empty_like(models)
        ptr, cells, w2 = self._graph
        _native.check(f._lib.adt_gn_regularize(
            f._plan, int(models.shape[0]), f.C, _native.ptr(ptr), _native.ptr(cells), _native.ptr(w2),
            float(s.regularization), float(s.temporal_regularization), _native.ptr(models.contiguous()),
            _native.ptr(out), f._stream()), f._plan, "adt_gn_regularize")
        return out

    def quadratic(self, models, step, residual0, residual1) -> tuple[float, float, float]:
        """(a0, a1, a2) of phi(tau) along ``step``: weighted data residuals at tau = 0 and their
        change to the candidate (``residual1``), and the regularization of models and step."""

        gm, gs = self.regularized(models), self.regularized(step)
        values = torch.stack([
            (residual0 * residual0).sum() + (models * gm).sum(),
            (residual0 * residual1).sum() + (step * gm).sum(),
            (residual1 * residual1).sum() + (step * gs).sum(),
        ]).cpu().numpy()
        return float(values[0]), float(values[1]), float(values[2])

    def objective(self, models: Tensor, predicted: Tensor, observed: Tensor, weights: Tensor) -> Tensor:
        """Data misfit plus regularization at ``models`` (device scalar)."""

        residual = weights * (predicted - observed)
        return (residual * residual).sum() + (models * self.regularized(models)).sum()

    # ---------------------------------------------------------------- one window
    def invert_window(self, observed_log: Tensor, initial_log: Tensor, screen=None,
                      previous: Tensor | None = None) -> WindowResult:
        """Gauss-Newton iterations of one window (adtlert/inversion/core.py:81-300): observed
        ``(T, D)`` log data, initial ``(T, C)`` log models. With ``screen`` (a surrogate screen,
        see surrogate.py) the line search runs on the screen's predictions and only the accepted
        model is solved by the FEM, which falls back to the plain candidate evaluation whenever
        that model does not lower the objective; the screen may also start the window from
        ``previous`` (the preceding window's final models) instead of ``initial_log``."""

        s, f = self.settings, self.forward
        observed = observed_log.to(self.device, torch.float64)
        T = int(observed.shape[0])
        weights = torch.full((T, f.D), 1.0 / float(s.data_std), dtype=torch.float64, device=self.device)
        models = self._clip(initial_log.to(self.device, torch.float64)).contiguous()
        start, bound = (models, None) if screen is None else screen.window_start(self, observed, models, previous)
        predicted, J = self.linearize(start)
        warm = bound is not None
        if warm and float(self.objective(start, predicted, observed, weights)) > bound:
            screen.reject_start()  # the FEM does not confirm the screened start
            predicted, J = self.linearize(models)
            warm = False
        else:
            models = start
        stall = getattr(screen, "stall_tolerance", None) if warm else None
        decrease_tolerance = getattr(screen, "objective_tolerance", None) if warm else None
        cgls_iterations = getattr(screen, "cgls_iterations", None) if warm else None
        result = WindowResult(models, predicted, [])
        scale = max(math.sqrt(models.numel()), 1.0)
        for _ in range(s.max_iterations):
            residual0 = weights * (predicted - observed)
            delta = self.gauss_newton_step(J, weights, (-residual0).contiguous(), models, cgls_iterations)
            if s.max_log_step is not None:
                largest = float(delta.abs().max())
                if largest > s.max_log_step:
                    delta = delta * (s.max_log_step / largest)
            candidate = self._clip(models + s.step_length * delta).contiguous()
            step = candidate - models
            accepted = None
            decrease = None  # the step's predicted relative objective decrease (FEM line search)
            if screen is not None and s.line_search:
                accepted = screen.screened_step(self, models, step, candidate, predicted, observed, weights, result)
            if accepted is None:
                candidate_predicted, candidate_J = self.linearize(candidate)
                tau = 1.0
                if s.line_search:
                    residual1 = weights * (candidate_predicted - predicted)
                    a0, a1, a2 = self.quadratic(models, step, residual0, residual1)
                    tau = line_search_tau((a0, a1, a2))
                    decrease = -(2.0 * a1 * tau + a2 * tau * tau) / a0 if a0 > 0.0 else None
                    step = tau * step
                if tau < 0.95:
                    models = self._clip(models + step).contiguous()
                    predicted, J = self.linearize(models)
                else:
                    models, predicted, J = candidate, candidate_predicted, candidate_J
            else:
                tau, step, models, predicted, J = accepted
            result.taus.append(tau)
            residual = weights * (predicted - observed)
            chi2, step_sq, error = torch.stack([(residual * residual).mean(), (step * step).sum(),
                                                self._cgls_state()[2].double()]).cpu().tolist()
            self._check_cgls(error)
            result.chi2.append(chi2)
            if s.target_chi2 is not None and chi2 < s.target_chi2:
                result.stop_reason = "target_chi2"
                break
            if math.sqrt(step_sq) / scale < s.step_tolerance:
                result.stop_reason = "step_tolerance"
                break
            if stall is not None and len(result.chi2) >= 2 and \
                    abs(result.chi2[-1] - result.chi2[-2]) <= stall * result.chi2[-2]:
                result.stop_reason = "chi2_stalled"  # warm-started windows only (see SurrogateScreen)
                screen.counts["stalled_windows"] += 1
                break
            if decrease_tolerance is not None and decrease is not None and len(result.chi2) >= 2 and \
                    decrease < decrease_tolerance:
                result.stop_reason = "objective_converged"  # warm-started windows only (see SurrogateScreen)
                screen.counts["converged_windows"] += 1
                break
        result.log_models, result.predicted_log = models, predicted
        return result

    # ---------------------------------------------------------------- all windows
    def run(self, observed_log, initial_log, *, window_size: int = 3, window_step: int = 1, screen=None,
            windows: list[int] | None = None) -> TimeLapseResult:
        """Sliding-window inversion of ``(S, D)`` observed log data from ``(S, C)`` initial log
        models (adtlert/inversion/core.py:445-577). ``windows`` restricts the run to those window
        indices (a share of the windows when ranks split them); the combined models then cover
        only the steps those windows contain."""

        observed = torch.as_tensor(observed_log, dtype=torch.float64, device=self.device)
        initial = torch.as_tensor(initial_log, dtype=torch.float64, device=self.device)
        steps = int(observed.shape[0])
        starts = window_starts(steps, window_size, window_step)
        chosen = range(len(starts)) if windows is None else windows
        total = torch.zeros_like(initial)
        count = torch.zeros(steps, dtype=torch.float64, device=self.device)
        reports = []
        previous, previous_start = None, None
        for index in chosen:
            start = starts[index]
            end = start + window_size
            warm = previous if previous_start == start - 1 else None
            window = self.invert_window(observed[start:end], initial[start:end], screen, warm)
            previous, previous_start = window.log_models, start
            total[start:end] += window.log_models
            count[start:end] += 1.0
            reports.append({"window": index, "start": start, "iterations": len(window.chi2),
                            "final_chi2": window.chi2[-1] if window.chi2 else None, "stop": window.stop_reason,
                            "screened": window.screened, "fallbacks": window.fallbacks})
        covered = count > 0
        final = torch.where(covered[:, None], total / count.clamp(min=1.0)[:, None], initial)
        return TimeLapseResult(final, covered, reports)


def window_starts(steps: int, window_size: int, window_step: int = 1) -> list[int]:
    """Start of every window (adtlert/inversion/core.py:433-442): every ``window_step``-th start
    plus the last full window."""

    if window_size > steps:
        raise ValueError(f"window_size={window_size} exceeds n_times={steps}")
    starts = list(range(0, steps - window_size + 1, max(1, int(window_step))))
    return sorted(set(starts + [steps - window_size]))


@dataclass
class TimeLapseResult:
    final_log_models: Tensor  # (S, C): mean of the windows' log models per step
    covered: Tensor           # (S,) steps some inverted window contains
    windows: list[dict]


def window_share(count: int, rank: int, world: int) -> list[int]:
    """Window indices of ``rank`` when ``world`` ranks split ``count`` independent windows:
    contiguous, as equal as possible, every window in exactly one share."""

    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    short, longer = divmod(int(count), int(world))
    start = rank * short + min(rank, longer)
    return list(range(start, start + short + (1 if rank < longer else 0)))
