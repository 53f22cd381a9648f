"""Generate the golden vectors that pin the CPU oracle to AD-TLERT's own implementation.

This script runs the reference package (``adtlert``, from the AD-TLERT project root named by
the ``ADTLERT_REFERENCE`` environment variable) on the CPU with three substitutions that leave
its arithmetic untouched:

1. its CUDA device constant is replaced by ``cpu`` (every torch op then runs on the host);
2. the cuDSS batched solve (``adtlert/forward/cudss.py:63-122``) is replaced by SciPy's
   ``splu`` on the same CSR values, solved in the operator's precision;
3. the NVRTC sensitivity kernel (``adtlert/forward/kernels.py:222-268``) is replaced by the
   einsum the reference's own test compares that kernel against
   (``tests/test_kernels_gpu.py:24-29``).

``meshio`` is only used by the reference for file I/O (``adtlert/mesh/core.py:632-645``); a
stub module stands in for it. Each precision runs in its own interpreter because the
reference fixes ``FLOAT_DTYPE`` at import (``adtlert/utils/dtypes.py:10-23``).

Usage: ``ADTLERT_REFERENCE=<AD-TLERT project root> python tests/golden/make_golden.py`` (writes
``tests/golden/*.npz``).
"""

from __future__ import annotations

import os
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REFERENCE = Path(os.environ.get("ADTLERT_REFERENCE", ""))

sys.path.insert(0, str(HERE))
from cases import CASES, CASES3D, case3d_inputs, case_inputs  # noqa: E402


def _stub_meshio(directory: Path) -> None:
    package = directory / "meshio"
    package.mkdir(parents=True, exist_ok=True)
    (package / "__init__.py").write_text(
        "class Mesh:\n    pass\n\n\ndef read(path):\n    raise NotImplementedError('file I/O is not used')\n"
    )


def _patch_reference():
    import numpy as np
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    import torch

    torch.cuda.is_available = lambda: True
    import adtlert.forward.cudss as cudss

    cudss.CUDA = torch.device("cpu")
    import adtlert.forward.ert2p5d as e2
    import adtlert.forward.ert3d as e3
    import adtlert.forward.kernels as kernels

    e2._CUDA = torch.device("cpu")
    e3._CUDA = torch.device("cpu")

    def solve(self, key, pattern, values, rhs, *, spd, refactorize=True, factorization=None):
        dtype = values.dtype
        out = torch.empty(rhs.shape, dtype=dtype)
        np_dtype = np.float64 if dtype == torch.float64 else np.float32
        for b in range(values.shape[0]):
            matrix = sp.csr_matrix(
                (values[b].numpy().astype(np_dtype), pattern.indices, pattern.indptr),
                shape=pattern.shape,
            ).tocsc()
            lu = spl.splu(matrix)
            out[b] = torch.as_tensor(lu.solve(rhs[b].numpy().astype(np_dtype).T).T, dtype=dtype)
        return out

    cudss.BatchedSolver.solve = solve

    def sensitivity(phi, a, b, m, n, cells, templates):
        phi = torch.cat((phi, phi.new_zeros(phi.shape[0], 1, phi.shape[2])), 1)
        current = (phi[:, a] - phi[:, b])[..., cells]
        receiver = (phi[:, m] - phi[:, n])[..., cells]
        return -torch.einsum("wdci,wcij,wdcj->dc", receiver, templates.to(phi.dtype), current)

    e2.normal_sensitivity = sensitivity
    kernels.normal_sensitivity = sensitivity
    e3.normal_sensitivity = sensitivity
    return e2, e3


def _run_2p5d(name: str, spec: dict, precision: str) -> dict:
    import numpy as np
    import torch

    e2, _ = _patch_reference()
    from adtlert.mesh import Mesh
    from adtlert.survey import Survey

    inputs = case_inputs(name)
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"], surface_node_ids=inputs.get("surface_node_ids"))
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = e2.ERTForward2p5D.from_mesh_survey(
        mesh, survey, topographic_geometric_factor_mode=inputs.get("gf_mode", "analytic")
    )
    dtype = forward.dtype
    sigma = torch.as_tensor(inputs["sigma"], dtype=dtype)
    cotangent = torch.as_tensor(inputs["cotangent"], dtype=dtype)
    direction = torch.as_tensor(inputs["direction"], dtype=dtype)
    response = forward.solve(sigma)
    fields = forward._fields(sigma).total
    out = {
        "wavenumbers": forward.wavenumbers.numpy(),
        "weights": forward.weights.numpy(),
        "geometric_factors": forward._geometric_factors().numpy(),
        "apparent_resistivity": response.apparent_resistivity.numpy(),
        "resistance": response.resistance.numpy(),
        "electrode_potentials": response.electrode_potentials.numpy(),
        "nnz": np.asarray(forward.discretization.pattern.nnz),
        "jacobian": forward.jacobian(sigma).numpy(),
        "vjp": forward.vjp(sigma, cotangent).numpy(),
        "jvp": forward.jvp(sigma, direction).numpy(),
        "normal_vjp": forward.normal_vjp(sigma, cotangent).numpy(),
        "normal_jvp": forward.normal_jvp(sigma, direction).numpy(),
        "homogeneous_apparent_resistivity": forward.apparent_resistivity_values(
            torch.full((mesh.cell_count,), 0.01, dtype=dtype)
        ).numpy(),
    }
    if precision == "float64" and not forward.use_numerical_primary:
        out["total_fields"] = fields.numpy()
    if forward.use_numerical_primary:
        out["integrated_potentials"] = response.integrated_potentials.numpy()
        out["discretization_nodes"] = np.asarray(forward.discretization.dof_nodes, dtype=np.float64)
    chunked = forward.jacobian(sigma, batch_size=5).numpy()
    assert np.allclose(chunked, out["jacobian"], rtol=1e-5, atol=1e-6 * np.abs(chunked).max())
    if spec.get("exact_jacobian"):
        out["jacobian_exact"] = forward.jacobian(
            sigma, include_robin_boundary_derivative=True, normal_sensitivity=False
        ).numpy()
    ids = inputs.get("parameter_ids")
    if ids is not None:
        count = int(ids.max()) + 1
        _, aggregated = forward.solve_with_jacobian(
            sigma, jacobian_cell_parameter_ids=ids, jacobian_parameter_count=count
        )
        out["jacobian_parameters"] = aggregated.numpy()
        out["normal_vjp_parameters"] = forward.normal_vjp(
            sigma, cotangent, cell_parameter_ids=ids, parameter_count=count
        ).numpy()
    return out


def _run_3d(name: str, precision: str) -> dict:
    import numpy as np
    import torch

    _, e3 = _patch_reference()
    from adtlert.mesh import Mesh3D
    from adtlert.survey import Survey

    inputs = case3d_inputs(name)
    mesh = Mesh3D.from_arrays(inputs["nodes"], inputs["cells"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    forward = e3.ERTForward3D.from_mesh_survey(mesh, survey, boundary_mode=inputs["boundary"],
                                               element_order=inputs["order"])
    sigma = torch.as_tensor(inputs["sigma"], dtype=torch.float64)
    cotangent = torch.as_tensor(inputs["cotangent"], dtype=torch.float64)
    direction = torch.as_tensor(inputs["direction"], dtype=torch.float64)
    response = forward.solve(sigma)
    out = {
        "geometric_factors": forward._geometric_factors().numpy(),
        "apparent_resistivity": response.apparent_resistivity.numpy(),
        "resistance": response.resistance.numpy(),
        "node_potentials": response.node_potentials.numpy(),
        "jacobian": forward.jacobian(sigma).numpy(),
        "jacobian_robin": forward.jacobian(sigma, include_robin_boundary_derivative=True).numpy(),
        "vjp": forward.vjp(sigma, cotangent).numpy(),
        "jvp": forward.jvp(sigma, direction).numpy(),
        "normal_vjp": forward.normal_vjp(sigma, cotangent).numpy(),
        "normal_jvp": forward.normal_jvp(sigma, direction).numpy(),
        "homogeneous_apparent_resistivity": forward.apparent_resistivity_values(
            torch.full((mesh.cell_count,), 0.01, dtype=torch.float64)
        ).numpy(),
    }
    return out


def _child(name: str, precision: str, target: str) -> None:
    import numpy as np

    sys.path.insert(0, str(REFERENCE))
    out = _run_3d(name, precision) if name in CASES3D else _run_2p5d(name, CASES[name], precision)
    np.savez_compressed(target, **out)


def main() -> None:
    if len(sys.argv) == 4 and sys.argv[1] == "--child":
        _, _, name, precision = sys.argv
        _child(name, precision, os.environ["GOLDEN_TARGET"])
        return
    if not (REFERENCE / "adtlert").is_dir():
        raise SystemExit("set ADTLERT_REFERENCE to the AD-TLERT project root (the folder holding adtlert/)")
    with tempfile.TemporaryDirectory() as stub:
        _stub_meshio(Path(stub))
        only = sys.argv[1:]
        for name in [*CASES, *CASES3D]:
            if only and name not in only:
                continue
            for precision in ("float64", "float32"):
                target = HERE / f"{name}_{precision}.npz"
                env = dict(os.environ)
                env["PYTHONPATH"] = os.pathsep.join((stub, str(REFERENCE), str(HERE)))
                env["ADTLERT_ENABLE_FLOAT64"] = "1" if precision == "float64" else "0"
                env["GOLDEN_TARGET"] = str(target)
                env["OMP_NUM_THREADS"] = "1"
                subprocess.run(
                    [sys.executable, __file__, "--child", name, precision],
                    check=True,
                    env=env,
                )
                print("wrote", target.name, f"{target.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
