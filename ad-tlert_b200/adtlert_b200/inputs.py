"""Validation of models, cotangents and parameter maps (same messages and exception types as
adtlert/forward/inputs.py:13-100)."""

from __future__ import annotations

import numpy as np
import torch

FLOAT_DTYPE = torch.float32
"""Result dtype. Fields and Jacobians are computed in float32 on the GPU (the direct solver
factorizes in float64); the reference's optional float64 mode is not provided."""

Tensor = torch.Tensor


def _host(values: Tensor):
    """NumPy view of a CPU float tensor (checks on it avoid torch's per-op overhead), else None."""

    return values.detach().numpy() if values.device.type == "cpu" else None


def _all_finite(values: Tensor) -> bool:
    host = _host(values)
    return bool(np.isfinite(host).all()) if host is not None else bool(torch.isfinite(values).all())


def _any_nonpositive(values: Tensor) -> bool:
    host = _host(values)
    return bool((host <= 0.0).any()) if host is not None else bool(torch.any(values <= 0.0))


def check_finite(values: Tensor, context: str) -> None:
    if not bool(torch.isfinite(values).all()):
        raise FloatingPointError(f"{context} produced non-finite values")


def finite_flag(values: Tensor) -> Tensor:
    """A one-element boolean on ``values``' device, True iff every entry is finite, computed in
    one read with no full-size temporary: the minimum and maximum are finite exactly when every
    entry is (min/max propagate NaN, and an infinite entry is an extreme)."""

    if values.numel() == 0:
        return torch.ones((), dtype=torch.bool, device=values.device)
    low, high = torch.aminmax(values)
    return torch.isfinite(low) & torch.isfinite(high)


def cell_vector(values, count: int, dtype: torch.dtype = FLOAT_DTYPE) -> Tensor:
    vector = torch.as_tensor(values, dtype=dtype)
    if vector.ndim == 0:
        vector = vector.expand(count)
    elif vector.shape != (count,):
        raise ValueError(f"conductivity must be scalar or shape ({count},)")
    if not _all_finite(vector):
        raise ValueError("conductivity must contain finite values")
    return vector


def conductivity_model(values, count: int, dtype: torch.dtype = FLOAT_DTYPE) -> Tensor:
    model = cell_vector(values, count, dtype)
    if _any_nonpositive(model):
        raise ValueError("conductivity must contain positive finite values")
    return model


def conductivity_series(values, count: int, dtype: torch.dtype = FLOAT_DTYPE) -> Tensor:
    models = torch.as_tensor(values, dtype=dtype)
    if models.ndim != 2 or models.shape[1] != count:
        raise ValueError(f"conductivities must have shape (n_steps, {count})")
    if not _all_finite(models) or _any_nonpositive(models):
        raise ValueError("conductivity must contain positive finite values")
    return models


def measurement_vector(values, count: int, dtype: torch.dtype) -> Tensor:
    vector = torch.as_tensor(values, dtype=dtype)
    if vector.ndim == 0:
        return vector.expand(count)
    if vector.shape != (count,):
        raise ValueError(f"cotangent must be scalar or shape ({count},)")
    return vector


def cotangent_series(values, steps: int, count: int) -> Tensor:
    cotangents = torch.as_tensor(values, dtype=FLOAT_DTYPE)
    if tuple(cotangents.shape) != (steps, count):
        raise ValueError(f"cotangents must have shape {(steps, count)}")
    return cotangents


def parameter_targets(cell_parameter_ids, parameter_count, cell_count: int) -> tuple[np.ndarray, int]:
    """Output column of every cell (-1: dropped) and the number of columns."""

    if cell_parameter_ids is None:
        if parameter_count is not None:
            raise ValueError("parameter_count requires cell_parameter_ids")
        return np.arange(cell_count, dtype=np.int64), cell_count
    if isinstance(cell_parameter_ids, Tensor):
        cell_parameter_ids = cell_parameter_ids.cpu()
    ids = np.asarray(cell_parameter_ids).astype(np.int64).reshape(-1)
    if ids.shape != (cell_count,):
        raise ValueError(f"cell_parameter_ids must have shape ({cell_count},)")
    if np.any(ids < -1) or not np.any(ids >= 0):
        raise ValueError("cell_parameter_ids may only contain -1 or non-negative ids, with at least one active")
    count = int(ids.max()) + 1 if parameter_count is None else int(parameter_count)
    if count <= int(ids.max()):
        raise ValueError("parameter_count is smaller than the largest cell parameter id")
    return ids, count


def option(value: str, choices: tuple[str, ...], name: str) -> str:
    normalized = str(value).strip().lower()
    if normalized not in choices:
        raise ValueError(f"{name} must be one of: {', '.join(sorted(choices))}")
    return normalized
