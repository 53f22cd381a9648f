"""The launch-shape autotuner (``adt_autotune``): it picks a setting for every plan shape, the
operator's results after tuning still meet the FP64 oracle, a saved choice round-trips, and
out-of-range settings are refused with the reference's ValueError."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, ERTForward3D, Mesh, Mesh3D, Survey, synthetic
from cases import box_tetrahedra, case_inputs, structured_section
from conftest import assert_close

pytestmark = pytest.mark.gpu

TOL = 1e-4
KERNELS = {"direct", "tc_pipelined", "tc", "fma"}


def _checked(forward, sigma, oracle_jacobian, oracle_resistance, tiled: bool, kernels: set):
    s32 = torch.as_tensor(sigma, dtype=torch.float32)
    before = forward.jacobian(s32)
    chosen = forward.autotune(s32, repeats=2)
    assert chosen["strip_fill"] in (1, 2, 4, 8)
    assert chosen["split_fill"] in ((0, 1, 2) if tiled else (2,))
    assert chosen["jacobian_kernel"] in kernels
    assert chosen["fields_ms"] > 0.0 and chosen["jacobian_ms"] > 0.0
    saved = forward.tuning()
    assert saved == {k: chosen[k] for k in ("strip_fill", "split_fill", "jacobian_kernel")}
    # the tuning run used a factor slot: a later call must refactorize its own model
    other = s32 * 1.5
    assert_close(forward.resistance(other), oracle_resistance(sigma * 1.5), TOL, "resistance after tuning")
    after = forward.jacobian(s32)
    assert_close(after, oracle_jacobian(sigma), TOL, "jacobian after tuning")
    assert_close(after, before, 1e-5, "jacobian before and after tuning")
    forward.set_tuning(saved)
    assert forward.tuning() == saved
    with pytest.raises(ValueError, match="tuning out of range"):
        forward.set_tuning(dict(saved, strip_fill=3))
    return chosen


def test_autotune_flat_section():
    from oracle.ert2p5d import Oracle2p5D

    inputs = case_inputs("tri_flat")
    forward = ERTForward2p5D(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                             Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    oracle = Oracle2p5D(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"])
    chosen = _checked(forward, inputs["sigma"], oracle.normal_jacobian, oracle.resistance, False,
                      {"tc_pipelined", "tc", "fma"})
    assert chosen["jacobian_kernel"] != "direct"  # 17 wavenumbers: the direct form does not apply


def test_autotune_tiled_section():
    from oracle.ert2p5d import Oracle2p5D

    xs = np.linspace(0.0, 40.0, 81)
    depths = np.concatenate((np.linspace(0.0, 10.0, 41), np.linspace(10.5, 30.0, 30)))
    nodes, cells = structured_section(xs, depths)
    electrodes = np.column_stack((np.linspace(4.0, 36.0, 17), np.zeros(17)))
    measurements = synthetic.dipole_dipole(17, 2, 4)
    forward = ERTForward2p5D(Mesh.from_arrays(nodes, cells), Survey.from_arrays(electrodes, measurements))
    assert forward.plan_info["max_block"] > 64
    sigma = np.exp(np.random.default_rng(8).normal(np.log(0.01), 0.5, len(cells)))
    oracle = Oracle2p5D(nodes, cells, electrodes, measurements)
    _checked(forward, sigma, oracle.normal_jacobian, oracle.resistance, True, {"tc_pipelined", "tc", "fma"})


def test_autotune_box():
    from oracle.ert3d import Oracle3D

    nodes, cells = box_tetrahedra(nx=9, ny=8, nz=8)
    top = np.flatnonzero(np.isclose(nodes[:, 2], 0.0) & np.isclose(nodes[:, 1], 6.0))
    electrodes = nodes[top[np.argsort(nodes[top, 0])]]
    count = len(electrodes)
    measurements = np.asarray([(i, i + 1, i + 1 + n, i + 2 + n) for n in (1, 2) for i in range(count)
                               if i + 2 + n < count])
    forward = ERTForward3D(Mesh3D.from_arrays(nodes, cells), Survey.from_arrays(electrodes, measurements))
    sigma = np.exp(np.random.default_rng(9).normal(np.log(0.01), 0.5, len(cells)))
    oracle = Oracle3D(nodes, cells, electrodes, measurements)
    tiled = forward.plan_info["max_block"] > 64
    _checked(forward, sigma, lambda s: oracle.jacobian(s, False), oracle.resistance, tiled, KERNELS)
