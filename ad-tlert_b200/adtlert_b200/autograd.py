"""Differentiable apparent resistivity over this library's operators.

Observable contract of the reference bridge (adtlert/forward/autograd.py:17-207), kept as is:
``apparent_resistivity_autograd(conductivity, forward_operator, currents=1.0)`` takes one model
``(cells,)`` or a series ``(steps, cells)``, returns ``k R / I`` on the conductivity's device
and dtype, back-propagates to the conductivity and to scalar, one-element or per-datum currents
(once differentiable), supports forward-mode AD, and raises the same TypeError / ValueError
messages for bad arguments.

How it gets there is this library's: a conductivity that lives on the GPU stays there. Its
resistances, the adjoint (exact VJP, reusing the forward factorization; no Jacobian is formed)
and the tangents come from the operator's device-resident entry points, so neither the model,
nor the resistances, nor the gradient crosses to the host. A CPU conductivity goes through the
operator's public methods, whose results are CPU tensors, exactly like the reference's path.
"""

from __future__ import annotations

from typing import Any

import torch
from torch.autograd.function import once_differentiable

from .ert2p5d import ERTForward2p5D
from .ert3d import ERTForward3D
from .inputs import FLOAT_DTYPE

Tensor = torch.Tensor


def _checked(conductivity, currents, operator) -> None:
    """The reference's argument checks, with its exception types and messages."""

    if not isinstance(operator, (ERTForward2p5D, ERTForward3D)):
        raise TypeError("forward_operator must be an ERTForward2p5D or ERTForward3D instance")
    if not isinstance(conductivity, Tensor) or not conductivity.is_floating_point():
        raise TypeError("conductivity must be a floating-point torch.Tensor")
    cells, data = operator.C, operator.D
    if conductivity.ndim not in (1, 2) or conductivity.shape[-1] != cells:
        raise ValueError(
            f"conductivity must have shape ({cells},) or (n_steps, {cells}), got {tuple(conductivity.shape)}")
    low, high = torch.aminmax(conductivity.detach())
    if not (bool(torch.isfinite(low)) and bool(torch.isfinite(high))) or float(low) <= 0.0:
        raise ValueError("conductivity must contain finite positive values")
    if not isinstance(currents, Tensor) or not currents.is_floating_point():
        raise TypeError("currents must be a floating-point torch.Tensor")
    if tuple(currents.shape) not in {(), (1,), (data,)}:
        raise ValueError(f"currents must be scalar or have shape ({data},), got {tuple(currents.shape)}")
    if not bool(torch.isfinite(currents).all()) or bool((currents == 0.0).any()):
        raise ValueError("currents must contain finite non-zero values")


class _Evaluation:
    """Where one call's arithmetic happens: the operator's GPU for CUDA conductivities, the host
    (through the public CPU methods) otherwise."""

    def __init__(self, operator, on_gpu: bool) -> None:
        self.operator = operator
        self.on_gpu = on_gpu
        self.device = operator.device if on_gpu else torch.device("cpu")

    def models(self, conductivity: Tensor) -> Tensor:
        series = conductivity.detach().reshape(-1, self.operator.C)
        return series.to(self.device, FLOAT_DTYPE).contiguous()

    def factors(self) -> Tensor:
        return self.operator._geometric_factors().to(self.device)

    def resistances(self, models: Tensor) -> Tensor:
        if self.on_gpu:
            return self.operator._resistances_device(models)
        return self.operator.resistance_series(models)

    def vjp(self, models: Tensor, cotangents: Tensor) -> Tensor:
        if self.on_gpu:
            return self.operator._vjp_device(models, cotangents)
        return self.operator.vjp_series(models, cotangents)

    def jvp(self, model: Tensor, direction: Tensor) -> Tensor:
        if self.on_gpu:
            return self.operator._jvp_device(model, direction)
        return self.operator.jvp(model, direction)


def _current_gradient(per_datum: Tensor, shape: torch.Size) -> Tensor:
    """Gradient of the currents from the per-datum gradient, reduced to the currents' shape."""

    if tuple(shape) == (1,):
        return per_datum.sum().reshape(1)
    if len(shape) == 0:
        return per_datum.sum()
    return per_datum


class ERT2p5DApparentResistivityFunction(torch.autograd.Function):
    """Apparent resistivity of one model ``(cells,)`` or a series ``(steps, cells)``, for a 2.5D
    or a 3D operator."""

    @staticmethod
    def forward(ctx: Any, conductivity, currents, forward_operator):
        _checked(conductivity, currents, forward_operator)
        run = _Evaluation(forward_operator, conductivity.is_cuda)
        models = run.models(conductivity)
        resistance = run.resistances(models)
        factors = run.factors().to(resistance.dtype)
        current = currents.detach().to(run.device, resistance.dtype)
        apparent = factors * resistance / current
        ctx.run = run
        ctx.input_shape, ctx.input_kind = conductivity.shape, (conductivity.device, conductivity.dtype)
        ctx.current_shape, ctx.current_kind = currents.shape, (currents.device, currents.dtype)
        kept = (models, current, apparent, factors)
        ctx.save_for_backward(*kept)
        ctx.save_for_forward(*kept)
        device, dtype = ctx.input_kind
        return apparent.reshape(*conductivity.shape[:-1], -1).to(device=device, dtype=dtype)

    @staticmethod
    @once_differentiable
    def backward(ctx: Any, grad_output):
        models, current, apparent, factors = ctx.saved_tensors
        upstream = grad_output.detach().reshape(apparent.shape).to(apparent.device, apparent.dtype)
        conductivity_grad = currents_grad = None
        if ctx.needs_input_grad[0]:
            gradient = ctx.run.vjp(models, upstream * factors / current)
            device, dtype = ctx.input_kind
            conductivity_grad = gradient.reshape(ctx.input_shape).to(device=device, dtype=dtype)
        if ctx.needs_input_grad[1]:
            per_datum = (-upstream * apparent / current).sum(dim=0)
            device, dtype = ctx.current_kind
            currents_grad = _current_gradient(per_datum, ctx.current_shape).to(device=device, dtype=dtype)
        return conductivity_grad, currents_grad, None

    @staticmethod
    def jvp(ctx: Any, conductivity_tangent, currents_tangent, forward_operator_tangent):
        del forward_operator_tangent
        models, current, apparent, factors = ctx.saved_tensors
        run = ctx.run
        tangent = torch.zeros_like(apparent)
        if conductivity_tangent is not None:
            directions = conductivity_tangent.detach().reshape(models.shape).to(run.device, FLOAT_DTYPE)
            resistance_tangent = torch.stack([run.jvp(model, direction).to(run.device, apparent.dtype)
                                              for model, direction in zip(models, directions, strict=True)])
            tangent = tangent + factors * resistance_tangent / current
        if currents_tangent is not None:
            tangent = tangent - apparent * currents_tangent.detach().to(run.device, apparent.dtype) / current
        device, dtype = ctx.input_kind
        return tangent.reshape(*ctx.input_shape[:-1], -1).to(device=device, dtype=dtype)


ERT3DApparentResistivityFunction = ERT2p5DApparentResistivityFunction
ERTApparentResistivityFunction = ERT2p5DApparentResistivityFunction


def apparent_resistivity_autograd(conductivity, forward_operator, currents=1.0):
    """Differentiable apparent resistivity; the output is on the conductivity's device and dtype."""

    if not isinstance(conductivity, Tensor):
        raise TypeError("conductivity must be a torch.Tensor")
    currents = torch.as_tensor(currents, device=conductivity.device, dtype=conductivity.dtype)
    return ERT2p5DApparentResistivityFunction.apply(conductivity, currents, forward_operator)
