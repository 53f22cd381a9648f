"""Log-space response and Jacobian of an operator (adtlert/forward/modeling.py:137-162).

``d log(rhoa) / d log(rho) = k J_R (-sigma) / rhoa``: the row factor k / rhoa and the column
factor -sigma are applied by one kernel while the Jacobian is still on the device, and the
result is widened to float64 there a block of rows at a time, so only the final matrix crosses
to the host and the device never holds a whole float64 copy.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native
from .ert2p5d import _widened_to_host


def log_response_and_jacobian(operator, conductivity, *, chain=None, **solve_kwargs) -> tuple[np.ndarray, np.ndarray]:
    """``log(rhoa)`` and ``d log(rhoa) / d log(rho)`` from the explicit resistance Jacobian.

    ``chain`` is the conductivity of each Jacobian column (defaults to ``conductivity``); it
    differs when the operator aggregates columns into inversion parameters.
    """

    response, jacobian = operator._solve_with_jacobian_device(conductivity, **solve_kwargs)
    device = jacobian.device
    rhoa = response.apparent_resistivity.to(torch.float64)
    factors = torch.as_tensor(operator._geometric_factors(), dtype=torch.float64)
    row = (factors / rhoa).to(device).contiguous()
    column_values = conductivity if chain is None else chain
    column = -torch.as_tensor(column_values, dtype=torch.float64).reshape(-1).to(device).contiguous()
    rows, columns = int(jacobian.shape[0]), int(jacobian.shape[1])
    if column.numel() != columns:
        raise ValueError(f"chain must have {columns} entries, got {column.numel()}")
    jacobian = jacobian.contiguous()
    lib = _native.load_library()
    _native.check(lib.adt_scale_rows_columns(_native.ptr(jacobian), rows, columns, _native.ptr(row), _native.ptr(column),
                                             _native.stream_handle(device)), None, "adt_scale_rows_columns")
    # widened to float64 on the device (exact) in row blocks, so the host receives the final array
    return np.log(np.asarray(response.apparent_resistivity, dtype=float)), _widened_to_host(jacobian).numpy()
