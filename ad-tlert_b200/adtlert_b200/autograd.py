"""PyTorch autograd bridge (semantics of adtlert/forward/autograd.py:17-207).

Forward returns apparent resistivity on the input's device and dtype; backward calls the
operator's ``vjp_series`` (adjoint kernels reusing the forward factorization, no Jacobian is
formed); forward-mode AD calls ``jvp``. Gradients flow to the conductivity and to scalar or
per-datum currents; second derivatives are not supported.
"""

from __future__ import annotations

from typing import Any

import torch
from torch.autograd.function import once_differentiable

from .ert2p5d import ERTForward2p5D
from .ert3d import ERTForward3D
from .inputs import FLOAT_DTYPE


def _operators():
    return (ERTForward2p5D, ERTForward3D)


def _validate_inputs(conductivity, currents, forward_operator) -> None:
    if not isinstance(forward_operator, _operators()):
        raise TypeError("forward_operator must be an ERTForward2p5D or ERTForward3D instance")
    if not isinstance(conductivity, torch.Tensor) or not conductivity.is_floating_point():
        raise TypeError("conductivity must be a floating-point torch.Tensor")
    cells = forward_operator.C
    if conductivity.ndim not in (1, 2) or conductivity.shape[-1] != cells:
        raise ValueError(
            f"conductivity must have shape ({cells},) or (n_steps, {cells}), got {tuple(conductivity.shape)}"
        )
    if not bool(torch.all(torch.isfinite(conductivity))) or bool(torch.any(conductivity <= 0.0)):
        raise ValueError("conductivity must contain finite positive values")
    if not isinstance(currents, torch.Tensor) or not currents.is_floating_point():
        raise TypeError("currents must be a floating-point torch.Tensor")
    count = forward_operator.D
    if tuple(currents.shape) not in {(), (1,), (count,)}:
        raise ValueError(f"currents must be scalar or have shape ({count},), got {tuple(currents.shape)}")
    if not bool(torch.all(torch.isfinite(currents))) or bool(torch.any(currents == 0.0)):
        raise ValueError("currents must contain finite non-zero values")


def _reduce_current_gradient(gradient: torch.Tensor, shape: torch.Size) -> torch.Tensor:
    if len(shape) == 0:
        return gradient.sum()
    if tuple(shape) == (1,):
        return gradient.sum().reshape(shape)
    return gradient


class ERT2p5DApparentResistivityFunction(torch.autograd.Function):
    """Apparent resistivity of one model ``(n_cells,)`` or a series ``(n_steps, n_cells)``."""

    @staticmethod
    def forward(ctx: Any, conductivity, currents, forward_operator):
        _validate_inputs(conductivity, currents, forward_operator)
        conductivity_work = conductivity.detach().to(device="cpu", dtype=FLOAT_DTYPE)
        currents_work = currents.detach().to(device="cpu", dtype=FLOAT_DTYPE)
        geometric_scale = forward_operator._geometric_factors().detach()
        resistance = forward_operator.resistance_series(
            conductivity_work.reshape(-1, conductivity_work.shape[-1])
        ).reshape(*conductivity_work.shape[:-1], -1)
        apparent_resistivity = geometric_scale * resistance / currents_work
        ctx.forward_operator = forward_operator
        ctx.conductivity_device, ctx.conductivity_dtype = conductivity.device, conductivity.dtype
        ctx.currents_device, ctx.currents_dtype = currents.device, currents.dtype
        ctx.currents_shape = currents.shape
        saved = (conductivity_work, currents_work, apparent_resistivity, geometric_scale)
        ctx.save_for_backward(*saved)
        ctx.save_for_forward(*saved)
        return apparent_resistivity.to(device=conductivity.device, dtype=conductivity.dtype)

    @staticmethod
    @once_differentiable
    def backward(ctx: Any, grad_output):
        conductivity, currents, apparent_resistivity, geometric_scale = ctx.saved_tensors
        output_cotangent = grad_output.detach().to(device="cpu", dtype=FLOAT_DTYPE)
        conductivity_gradient = None
        if ctx.needs_input_grad[0]:
            resistance_cotangent = output_cotangent * geometric_scale / currents
            conductivity_gradient = ctx.forward_operator.vjp_series(
                conductivity.reshape(-1, conductivity.shape[-1]),
                resistance_cotangent.reshape(-1, resistance_cotangent.shape[-1]),
            ).reshape(conductivity.shape)
            conductivity_gradient = conductivity_gradient.to(device=ctx.conductivity_device, dtype=ctx.conductivity_dtype)
        currents_gradient = None
        if ctx.needs_input_grad[1]:
            expanded = -output_cotangent * apparent_resistivity / currents
            currents_gradient = _reduce_current_gradient(expanded.reshape(-1, expanded.shape[-1]).sum(0), ctx.currents_shape)
            currents_gradient = currents_gradient.to(device=ctx.currents_device, dtype=ctx.currents_dtype)
        return conductivity_gradient, currents_gradient, None

    @staticmethod
    def jvp(ctx: Any, conductivity_tangent, currents_tangent, forward_operator_tangent):
        del forward_operator_tangent
        conductivity, currents, apparent_resistivity, geometric_scale = ctx.saved_tensors
        tangent = torch.zeros_like(apparent_resistivity)
        if conductivity_tangent is not None:
            direction = conductivity_tangent.detach().to(device="cpu", dtype=FLOAT_DTYPE)
            resistance_tangent = torch.stack([
                ctx.forward_operator.jvp(model, step)
                for model, step in zip(
                    conductivity.reshape(-1, conductivity.shape[-1]),
                    direction.reshape(-1, conductivity.shape[-1]),
                    strict=True,
                )
            ]).reshape(apparent_resistivity.shape)
            tangent = tangent + geometric_scale * resistance_tangent / currents
        if currents_tangent is not None:
            current_direction = currents_tangent.detach().to(device="cpu", dtype=FLOAT_DTYPE)
            tangent = tangent - apparent_resistivity * current_direction / currents
        return tangent.to(device=ctx.conductivity_device, dtype=ctx.conductivity_dtype)


ERT3DApparentResistivityFunction = ERT2p5DApparentResistivityFunction
ERTApparentResistivityFunction = ERT2p5DApparentResistivityFunction


def apparent_resistivity_autograd(conductivity, forward_operator, currents=1.0):
    """Differentiable apparent resistivity; output on the conductivity's device and dtype."""

    if not isinstance(conductivity, torch.Tensor):
        raise TypeError("conductivity must be a torch.Tensor")
    current_tensor = torch.as_tensor(currents, device=conductivity.device, dtype=conductivity.dtype)
    return ERT2p5DApparentResistivityFunction.apply(conductivity, current_tensor, forward_operator)
