"""Coordinate-network (INR) physics over this library's operators.

The reference's INR trainer (adtlert/inr/train.py:516-709) maps a network's log-resistivities to
log apparent resistivities through ``matrix_free_log_rhoa_series`` (adtlert/inr/physics.py:70-89)
and back-propagates the misfit with the operator's exact VJP: no Jacobian is ever formed. The
same entry points are given here with the same names, argument meaning and exception types, so
that trainer runs on these operators unchanged. A CUDA log-resistivity stays on the GPU through
the forward fields, the adjoint and the gradient (``apparent_resistivity_autograd``'s device
path); only the network's own parameters live elsewhere.

Facades that extend a reduced parameter vector to the forward mesh (the reference's
``ParameterizedERTForward2p5D``) are recognised by their ``log_model_to_full`` method and a
``forward_operator`` attribute, without importing the reference's inversion package.
"""

from __future__ import annotations

from typing import Any

import numpy as np
import torch

from .autograd import apparent_resistivity_autograd
from .ert2p5d import ERTForward2p5D
from .ert3d import ERTForward3D


def forward_operator(forward: Any) -> ERTForward2p5D | ERTForward3D:
    """The 2.5D or 3D operator behind ``forward`` (itself, or its ``forward_operator``)
    (adtlert/inr/physics.py:21-31)."""

    if isinstance(forward, (ERTForward2p5D, ERTForward3D)):
        return forward
    operator = getattr(forward, "forward_operator", None)
    if isinstance(operator, (ERTForward2p5D, ERTForward3D)):
        return operator
    raise TypeError("INR physics requires an ADTLERT ERTForward2p5D or ERTForward3D operator")


def _conductivity(forward: Any, log_resistivity: torch.Tensor) -> torch.Tensor:
    """Float64 forward-mesh conductivities of ``(..., n_parameters)`` log-resistivities
    (adtlert/inr/physics.py:34-44): exp(-log rho), after the facade's extension to the mesh."""

    extend = getattr(forward, "log_model_to_full", None)
    if extend is not None and not isinstance(forward, (ERTForward2p5D, ERTForward3D)):
        return torch.exp(-extend(log_resistivity))
    if isinstance(forward, (ERTForward2p5D, ERTForward3D)) or hasattr(forward, "forward_operator"):
        return torch.exp(-log_resistivity.to(torch.float64))
    raise TypeError(
        "INR physics requires ERTForward2p5D, ERTForward3D, ERTForwardModeling, or "
        "ParameterizedERTForward2p5D")


def select_cuda_device(device: torch.device | str = "cuda") -> dict[str, Any]:
    """Make ``device`` the current CUDA device; returns its index and name
    (adtlert/inr/physics.py:47-56)."""

    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"INR inversion runs on CUDA devices, got {device}")
    index = device.index if device.index is not None else torch.cuda.current_device()
    torch.cuda.set_device(index)
    return {"gpu_device_index": index, "gpu_name": torch.cuda.get_device_name(index)}


def prepare_cuda_forward(forward: Any, parameter_log: np.ndarray, *,
                         device: torch.device | str = "cuda") -> dict[str, Any]:
    """Select the device and warm the operator's field cache and factorizations at
    ``parameter_log`` (adtlert/inr/physics.py:59-67)."""

    report = select_cuda_device(device)
    model = torch.as_tensor(np.asarray(parameter_log, dtype=float).reshape(-1))
    forward_operator(forward).prepare(_conductivity(forward, model), include_solver_state=True)
    return report


def matrix_free_log_rhoa_series(log_resistivity: torch.Tensor, forward: Any) -> torch.Tensor:
    """``(n_steps, n_parameters)`` log-resistivity -> ``(n_steps, n_data)`` log apparent
    resistivity, differentiable by the operator's exact VJP (adtlert/inr/physics.py:70-83).

    Every step's fields come from one batched factorization per ``series_batch_steps`` models and
    stay in the operator's field store, which the backward pass reuses (the store must hold at
    least ``n_steps`` entries for that). The result has the input's dtype and device.
    """

    operator = forward_operator(forward)
    rhoa = apparent_resistivity_autograd(_conductivity(forward, log_resistivity), operator)
    return torch.log(rhoa).to(log_resistivity.dtype)


def matrix_free_log_rhoa(log_resistivity: torch.Tensor, forward: Any) -> torch.Tensor:
    """Log apparent resistivity of one model, without a dense Jacobian
    (adtlert/inr/physics.py:86-89)."""

    return matrix_free_log_rhoa_series(log_resistivity[None, :], forward)[0]


__all__ = [
    "forward_operator",
    "matrix_free_log_rhoa",
    "matrix_free_log_rhoa_series",
    "prepare_cuda_forward",
    "select_cuda_device",
]
