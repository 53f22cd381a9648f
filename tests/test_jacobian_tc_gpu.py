"""The tensor-core (tcgen05) and direct-form Jacobians against the CUDA-core Gram kernel and the
FP64 oracle.

``ADTLERT_B200_JACOBIAN=fma`` at plan creation selects the CUDA-core Gram kernel and ``tc`` the
tensor cores wherever they apply; by default single-wavenumber (3D) operators take the direct
form. All must agree to float32 accuracy on 2.5D sections (12 and 48 electrodes) and 3D boxes."""

import os

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, ERTForward3D, Mesh, Mesh3D, Survey, _native, synthetic
from cases import case3d_inputs, case_inputs
from conftest import assert_close
from oracle.ert2p5d import Oracle2p5D

pytestmark = pytest.mark.gpu


def _with_choice(choice, make):
    os.environ["ADTLERT_B200_JACOBIAN"] = choice
    try:
        return make()
    finally:
        del os.environ["ADTLERT_B200_JACOBIAN"]


def _pair(make):
    return make(), _with_choice("fma", make)


def test_tensor_core_jacobian_matches_the_cuda_core_kernel_2p5d():
    inputs = case_inputs("tri_flat")
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    tc, fma = _pair(lambda: ERTForward2p5D(mesh, survey))
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    a, b = tc.jacobian(sigma), fma.jacobian(sigma)
    assert_close(a, b, 2e-6, "tcgen05 vs FMA jacobian")
    oracle = Oracle2p5D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])
    assert_close(a, oracle.normal_jacobian(inputs["sigma"]), 1e-4, "tcgen05 jacobian vs oracle")


def test_tensor_core_jacobian_on_the_benchmark_section():
    nodes, cells, electrodes, abmn = synthetic.flat_section()
    mesh, survey = Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, abmn)
    tc, fma = _pair(lambda: ERTForward2p5D(mesh, survey))
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 1), dtype=torch.float32)
    a, b = tc.jacobian(sigma), fma.jacobian(sigma)
    assert torch.isfinite(a).all()
    assert_close(a, b, 2e-6, "tcgen05 vs FMA jacobian (48 electrodes)")
    assert torch.equal(a, tc.jacobian(sigma)), "bitwise repeatable"


@pytest.mark.parametrize("name", ["tet_mixed", "tet_p2_mixed"])
def test_direct_and_tensor_core_jacobians_3d(name):
    inputs = case3d_inputs(name)
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    options = {"element_order": inputs["order"], "boundary_mode": inputs["boundary"]}
    make = lambda: ERTForward3D(mesh, survey, **options)  # noqa: E731
    direct, fma = _pair(make)
    tc = _with_choice("tc", make)
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float32)
    reference = fma.jacobian(sigma)
    assert_close(direct.jacobian(sigma), reference, 2e-6, f"direct vs FMA jacobian ({name})")
    assert_close(tc.jacobian(sigma), reference, 2e-6, f"tcgen05 vs FMA jacobian ({name})")
    # a row range takes the rows in their own order instead of the plan's sorted order
    fields = direct._fields(sigma)
    D, C = reference.shape
    start, count = D // 3, D - D // 3 - 1
    part = torch.full((count, C), float("nan"), device="cuda")
    direct._call("adt_normal_jacobian", _native.ptr(fields), start, count, _native.ptr(part), direct._stream())
    full = direct._jacobian_device(fields, False, None)
    assert torch.equal(part, full[start:start + count])


def test_tensor_core_jacobian_with_more_rows_than_the_offset_table():
    # 4 x 1232 = 4928 rows: more than the 4096 rows whose Gram offsets stay in shared memory
    nodes, cells, electrodes, abmn = synthetic.flat_section()
    abmn = np.concatenate([abmn, abmn[::-1], abmn, abmn[::-1]])
    mesh, survey = Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, abmn)
    tc, fma = _pair(lambda: ERTForward2p5D(mesh, survey))
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 2), dtype=torch.float32)
    a, b = tc.jacobian(sigma), fma.jacobian(sigma)
    assert a.shape[0] == 4928 and torch.isfinite(a).all()
    assert_close(a, b, 2e-6, "tcgen05 vs FMA jacobian (4928 rows)")
    n = len(abmn) // 4
    assert torch.equal(a[:n], a[2 * n:3 * n]) and torch.equal(a[n:2 * n], a[3 * n:])


def test_jacobian_to_host_in_column_chunks_is_the_device_jacobian():
    nodes, cells, electrodes, abmn = synthetic.flat_section()
    mesh, survey = Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, abmn)
    sigma = torch.as_tensor(synthetic.layered_model(nodes, cells, 3), dtype=torch.float32)
    for forward in _pair(lambda: ERTForward2p5D(mesh, survey)):
        fields = forward._fields(sigma)
        expected = forward._jacobian_device(fields).cpu()
        for chunks in (1, 3, 8, 1000):  # 1000 is capped at C / 64
            device = torch.full_like(expected, float("nan"), device="cuda")
            host = torch.full(tuple(expected.shape), float("nan"), pin_memory=True)
            forward._call("adt_normal_jacobian_to_host", _native.ptr(fields.total), _native.ptr(device),
                          _native.ptr(host), chunks, forward._stream())
            torch.cuda.current_stream().synchronize()
            assert torch.equal(host, expected), f"{chunks} chunks"
        assert torch.equal(forward.jacobian(sigma), expected)
