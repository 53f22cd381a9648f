"""Launch-shape autotuning of an operator's plan (``adt_autotune``).

The solver's substitution strips, the tiled solver's split depth and the Jacobian kernel are
picked by timing the real entry points on a model of the caller's choosing; the reference
leaves these choices to cuDSS and to its kernel's fixed launch geometry
(adtlert/forward/kernels.py:222-268), so this has no counterpart there. The choice is kept by
the plan; ``tuning``/``set_tuning`` read and restore it (for example from a saved run on the
same device and discretization).
"""

from __future__ import annotations

import ctypes

import torch

from . import _native


def autotune(operator, conductivity=None, repeats: int = 3, jacobian: bool = True) -> dict:
    """Time every candidate launch shape on ``conductivity`` (default: uniform 1 S/m) and keep
    the fastest; returns the chosen settings and their times (ms)."""

    sigma = torch.ones(operator.C) if conductivity is None else operator._sigma(conductivity)
    sig = sigma.to(operator.device, torch.float32).reshape(1, -1).contiguous()
    entry = operator._solver.lookup(1)
    columns = operator.columns if hasattr(operator, "columns") else operator.E
    fields = torch.empty((1, getattr(operator, "W", 1), operator.N, columns), dtype=torch.float32, device=operator.device)
    cells = getattr(operator, "Cd", operator.C)
    J = torch.empty((operator.D, cells), dtype=torch.float32, device=operator.device) if jacobian else None
    result = _native.Tuning()
    with torch.cuda.device(operator.device):
        operator._call("adt_autotune", entry["slot"], _native.ptr(sig), 1, _native.ptr(fields), _native.ptr(J),
                       int(repeats), ctypes.byref(result), operator._stream())
    entry["name"] = None  # the slot holds the tuning model, which no factorization name describes
    return result.as_dict()


def tuning(operator) -> dict:
    result = _native.Tuning()
    _native.check(operator._lib.adt_get_tuning(operator._plan, ctypes.byref(result)), operator._plan, "adt_get_tuning")
    out = result.as_dict()
    del out["fields_ms"], out["jacobian_ms"]
    return out


def set_tuning(operator, settings: dict) -> None:
    value = _native.Tuning(strip_fill=int(settings["strip_fill"]), split_fill=int(settings["split_fill"]),
                           jacobian_kernel=_native.JACOBIAN_KERNELS.index(settings["jacobian_kernel"]))
    _native.check(operator._lib.adt_set_tuning(operator._plan, ctypes.byref(value)), operator._plan, "adt_set_tuning")
