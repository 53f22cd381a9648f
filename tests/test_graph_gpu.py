"""Fresh-model Jacobians replayed from a captured CUDA graph equal the same launch chain run
uncaptured bit for bit, agree with the operator's ``jacobian()`` to rounding, count their kernels
like the uncaptured chain, and refuse to launch once the plan reallocated a workspace the graph
holds."""

import numpy as np
import pytest
import torch

from adtlert_b200 import ERTForward2p5D, ERTForward3D, Mesh, Mesh3D, Survey, _native
from cases import box_tetrahedra, case_inputs
from conftest import assert_close

pytestmark = pytest.mark.gpu


def _uncaptured(forward, graph, sigma):
    """The captured chain's entry points called one by one on a slot of their own."""

    slot = forward._solver.private()
    sig = sigma.to(forward.device, torch.float32).contiguous()
    fields, normal, J = torch.empty_like(graph.fields), torch.empty_like(graph.normal), torch.empty_like(graph.J)
    reciprocal = torch.empty_like(normal)
    s = forward._stream()
    forward._call("adt_factorize_fields", slot, _native.ptr(sig), 1, s)
    forward._call("adt_solve_fields", slot, _native.ptr(sig), 1, _native.ptr(fields), s)
    forward._call("adt_measure", _native.ptr(fields), 1, _native.ptr(normal), _native.ptr(reciprocal), None, s)
    forward._call("adt_normal_jacobian", _native.ptr(fields), 0, forward.D, _native.ptr(J), s)
    return J.cpu()


def _models(sigma, count, seed):
    rng = np.random.default_rng(seed)
    return [torch.as_tensor(sigma * rng.uniform(0.5, 2.0, sigma.shape), dtype=torch.float32) for _ in range(count)]


def test_flat_graph_equals_jacobian_and_counts_its_kernels():
    inputs = case_inputs("tri_flat")
    forward = ERTForward2p5D(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                             Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    graph = forward.jacobian_graph()
    assert graph.kernels > 20
    for i, sigma in enumerate(_models(inputs["sigma"], 3, 1)):
        before = forward.kernel_launches()
        J = graph(sigma if i % 2 == 0 else sigma.cuda()).cpu()
        assert forward.kernel_launches() - before == graph.kernels
        assert torch.equal(J, _uncaptured(forward, graph, sigma)), f"model {i}: graph and its chain differ"
        assert_close(J, forward.jacobian(sigma), 1e-6, f"model {i}: graph and jacobian()")
    # a series of more models grows the measurement's potential table: the graph must refuse
    forward.resistance_series(torch.stack(_models(inputs["sigma"], 9, 2)))
    with pytest.raises(ValueError, match="reallocated since the capture"):
        graph(inputs["sigma"])
    graph.close()
    again = forward.jacobian_graph()
    sigma = _models(inputs["sigma"], 1, 3)[0]
    assert_close(again(sigma).cpu(), forward.jacobian(sigma), 1e-6, "recreated graph and jacobian()")
    again.close()


def test_box_graph_equals_jacobian():
    nodes, cells = box_tetrahedra(nx=8, ny=4, nz=4)
    top = np.flatnonzero(np.isclose(nodes[:, 2], 0.0) & np.isclose(nodes[:, 1], 6.0))
    electrodes = nodes[top[np.argsort(nodes[top, 0])]]
    count = len(electrodes)
    measurements = np.asarray([(i, i + 1, i + 2, i + 3) for i in range(count) if i + 3 < count])
    forward = ERTForward3D(Mesh3D.from_arrays(nodes, cells), Survey.from_arrays(electrodes, measurements))
    graph = forward.jacobian_graph()
    for sigma in _models(np.full(len(cells), 0.01), 2, 4):
        J = graph(sigma).cpu()
        assert torch.equal(J, _uncaptured(forward, graph, sigma))
        assert_close(J, forward.jacobian(sigma), 1e-6, "graph and jacobian()")
    graph.close()
