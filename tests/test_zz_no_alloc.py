"""adt_measure_static: the measurement entry point that allocates no device memory.

It is for callers that may not call cudaMalloc while running, for example because another
allocator has reserved all GPU memory up front, or because a loop must not block on the
driver's allocator. Its scratch table is a fixed array compiled into the library. This file
is collected last so that a failure here cannot hide the rest of the suite; it must pass both
alone in a fresh process and after the other tests.
"""

import ctypes

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, _native
from cases import case_inputs

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same kernels, same order: the two entry points should agree to rounding


def _operator():
    inputs = case_inputs("tri_flat")
    forward = ERTForward2p5D.from_mesh_survey(
        Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
        Survey.from_arrays(inputs["electrodes"], inputs["measurements"]),
    )
    return inputs, forward


def _measure(forward, name, fields, models):
    normal = torch.empty((models, forward.D), dtype=torch.float64, device=forward.device)
    reciprocal = torch.empty_like(normal)
    if name == "adt_measure":
        status = forward._lib.adt_measure(forward._plan, _native.ptr(fields), models, _native.ptr(normal),
                                          _native.ptr(reciprocal), None, forward._stream())
    else:
        status = forward._lib.adt_measure_static(forward._plan, _native.ptr(fields), models, _native.ptr(normal),
                                                 _native.ptr(reciprocal), forward._stream())
    _native.check(status, forward._plan, name)
    torch.cuda.synchronize(forward.device)
    return normal.cpu().numpy(), reciprocal.cpu().numpy()


def test_static_measure_matches_the_allocating_entry_point_twice_in_a_row():
    inputs, forward = _operator()
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    for scale, models in ((1.0, 2), (0.5, 3)):  # two calls in a row, different contents and sizes
        series = torch.stack([sigma * scale * (1.0 + 0.1 * i) for i in range(models)])
        fields, _ = forward._fields_series(series)
        stacked = forward._stack(fields)
        expected = _measure(forward, "adt_measure", stacked, models)
        actual = _measure(forward, "adt_measure_static", stacked, models)
        for a, e in zip(actual, expected):
            error = np.abs(a - e).max() / np.abs(e).max()
            assert error <= TOL, f"static measure differs by {error:.2e}"


def test_static_measure_rejects_requests_beyond_its_table():
    inputs, forward = _operator()
    models = 65536 // (forward.E + 1) ** 2 + 1
    fields = torch.zeros((1, forward.W, forward.N, forward.E), dtype=torch.float32, device=forward.device)
    normal = torch.empty((models, forward.D), dtype=torch.float64, device=forward.device)
    status = forward._lib.adt_measure_static(forward._plan, _native.ptr(fields), models, _native.ptr(normal),
                                             _native.ptr(normal), forward._stream())
    assert status == _native.ADT_INVALID_ARG
    assert "exceeds the static table" in _native.last_error(forward._plan)
