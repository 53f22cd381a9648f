"""CPU checks of the input validation and finiteness helpers (adtlert/forward/inputs.py:13-100)."""

import numpy as np
import pytest
import torch

from adtlert_b200.inputs import cell_vector, check_finite, conductivity_model, finite_flag


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_finite_flag_detects_every_non_finite_kind(dtype):
    rng = np.random.default_rng(0)
    values = torch.as_tensor(rng.standard_normal((37, 53)), dtype=dtype)
    assert bool(finite_flag(values))
    big = torch.full((1000,), torch.finfo(dtype).max, dtype=dtype)
    assert bool(finite_flag(big))  # finite entries at the type's maximum do not overflow the check
    for bad in (float("inf"), float("-inf"), float("nan")):
        planted = values.clone()
        planted[17, 41] = bad
        assert not bool(finite_flag(planted))
    opposite = values.clone()
    opposite[0, 0], opposite[1, 1] = float("inf"), float("-inf")
    assert not bool(finite_flag(opposite))
    assert bool(finite_flag(torch.empty((0, 5), dtype=dtype)))


def test_finite_flag_at_the_float64_maximum():
    big = torch.full((4,), torch.finfo(torch.float64).max, dtype=torch.float64)
    assert bool(finite_flag(big))


def test_validation_messages():
    with pytest.raises(FloatingPointError, match="jacobian produced non-finite values"):
        check_finite(torch.tensor([1.0, float("nan")]), "jacobian")
    with pytest.raises(ValueError, match="finite"):
        cell_vector([1.0, float("inf")], 2)
    with pytest.raises(ValueError):
        conductivity_model([1.0, -1.0], 2)
