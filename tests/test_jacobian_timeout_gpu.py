"""Failure detection of the tensor-core Jacobian without a GPU fault.

The plan option adt_set_jacobian_wait_limit shortens the first wait of every block of
jacobian_tc_kernel (for its MMA chain) to one non-blocking poll, so the wait runs out while the
MMAs are still in flight: the blocks write NaN into their cells' columns, raise the plan's error
flag and still drain their own MMAs with the full bounded wait before freeing tensor memory. The
next call reports ADT_TIMEOUT (RuntimeError); restoring the default wait clears the flag and the
Jacobian is exact again."""

import pytest
import torch

from adtlert_b200 import ERTForward2p5D, Mesh, Survey, _native, synthetic

pytestmark = pytest.mark.gpu


def test_short_mma_wait_reports_a_timeout_and_recovers():
    nodes, cells, electrodes, rows = synthetic.flat_section()
    forward = ERTForward2p5D(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, rows))
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 2), dtype=torch.float32)
    fields = forward._fields(sigma).total
    lib, plan, stream = forward._lib, forward._plan, forward._stream()

    def jacobian():
        out = torch.empty((forward.D, forward.C), dtype=torch.float32, device="cuda")
        _native.check(lib.adt_normal_jacobian(plan, _native.ptr(fields), 0, forward.D, _native.ptr(out), stream), plan,
                      "adt_normal_jacobian")
        torch.cuda.synchronize()
        return out

    expected = jacobian()
    assert torch.isfinite(expected).all()
    _native.check(lib.adt_set_jacobian_wait_limit(plan, 1), plan, "adt_set_jacobian_wait_limit")
    timed_out = jacobian()
    assert torch.isnan(timed_out).any(), "no block gave up after one poll"
    with pytest.raises(RuntimeError, match="timed out"):
        jacobian()
    _native.check(lib.adt_set_jacobian_wait_limit(plan, 0), plan, "adt_set_jacobian_wait_limit")
    assert torch.equal(jacobian(), expected)
