"""Golden outputs of AD-TLERT's own windowed time-lapse inversion on a small seeded case.

Runs ``adtlert.inversion.invert_windowed_timelapse_log_resistivity`` (adtlert/inversion/
core.py:445-577) from the AD-TLERT project root named by ``ADTLERT_REFERENCE``, in the
reference's float64 mode, on the CPU, with the substitutions of ``make_golden.py`` (CPU device,
SciPy ``splu`` for the cuDSS solve, the reference test's einsum for the NVRTC kernel) plus one
more: its GPU CGLS (adtlert/inversion/optimizers.py:314-360) is given a torch namespace whose
tensors are created on the CPU, so the same statements run on the host. Inversion settings are
those of the reference's 363-window example (example/window_363/inversion_adtlert.py:483-603)
with 4 Gauss-Newton iterations; a second run records one iteration of the first window with a
20-iteration CGLS.

The case: the ``tri_flat`` section and survey of ``cases.py``, 5 time steps whose near-surface
resistivity drops step by step, data from the reference's own forward with 2 % multiplicative
noise, initial models the per-step median apparent resistivity (3 windows of 3 steps).

Usage: ``ADTLERT_REFERENCE=<AD-TLERT project root> python tests/golden/make_timelapse_golden.py``
(writes ``tests/golden/timelapse_small.npz``).
"""

from __future__ import annotations

import math
import os
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REFERENCE = Path(os.environ.get("ADTLERT_REFERENCE", ""))
TARGET = HERE / "timelapse_small.npz"
STEPS = 5
ITERATIONS = 4
DATA_STD = math.log1p(0.02)

sys.path.insert(0, str(HERE))
from cases import case_inputs  # noqa: E402


def series(inputs):
    """Seeded resistivity series (STEPS, cells): the case's model with a wetting front."""

    import numpy as np

    nodes, cells = inputs["nodes"], inputs["cells"]
    rho0 = 1.0 / np.asarray(inputs["sigma"], dtype=float)
    depth = nodes[:, 1].max() - nodes[cells].mean(axis=1)[:, 1]
    rng = np.random.default_rng(11)
    factor = rng.uniform(0.3, 0.7)
    out = []
    for t in range(STEPS):
        front = 4.0 * t / (STEPS - 1)
        out.append(np.where(depth < front, rho0 * factor, rho0))
    return np.stack(out)


def _child() -> None:
    import numpy as np
    import torch

    sys.path.insert(0, str(REFERENCE))
    from make_golden import _patch_reference

    e2, _ = _patch_reference()
    import adtlert.inversion.optimizers as optimizers
    from adtlert.inversion import InversionConfig, invert_windowed_timelapse_log_resistivity
    from adtlert.mesh import Mesh
    from adtlert.survey import Survey

    class HostTorch:
        """torch with tensors that would go to "cuda" created on the CPU."""

        def __getattr__(self, name):
            return getattr(torch, name)

        @staticmethod
        def as_tensor(*args, device=None, **kwargs):
            return torch.as_tensor(*args, **kwargs)

        @staticmethod
        def zeros(*args, device=None, **kwargs):
            return torch.zeros(*args, **kwargs)

    optimizers.torch = HostTorch()
    inputs = case_inputs("tri_flat")
    forward = e2.ERTForward2p5D.from_mesh_survey(Mesh.from_arrays(inputs["nodes"], inputs["cells"]),
                                                 Survey.from_arrays(inputs["electrodes"], inputs["measurements"]))
    rho = series(inputs)
    clean = np.stack([forward.apparent_resistivity_values(torch.as_tensor(1.0 / r, dtype=forward.dtype)).numpy()
                      for r in rho])
    noise = np.random.default_rng(12).standard_normal(clean.shape)
    observed = clean * np.exp(0.02 * noise)
    initial = np.tile(np.median(observed, axis=1)[None, :], (len(inputs["cells"]), 1))  # (cells, steps)
    config = InversionConfig(
        max_iterations=ITERATIONS, data_std=DATA_STD, data_misfit="weighted_log_l2", regularization=50.0,
        regularization_mode="model", temporal_regularization=10.0, temporal_regularization_type="temporal_smoothness",
        spatial_regularization="first_order_smoothness", optimization_algorithm="gauss_newton_cgls",
        linearized_solver="gpu_cgls", cgls_tolerance=1.0e-12, cgls_max_iterations=60, step_tolerance=1.0e-4,
        z_weight=1.0, model_bounds=(0.001, 1.0e4), max_log_step=None, line_search=True)
    result = invert_windowed_timelapse_log_resistivity(forward, observed, initial, window_size=3, window_step=1,
                                                       config=config)
    # one Gauss-Newton iteration of the first window with a 20-iteration CGLS: short enough that
    # the CGLS result does not depend on rounding, so it pins the linearized system tightly
    import dataclasses

    import adtlert.inversion.core as core

    short = dataclasses.replace(config, max_iterations=1, cgls_max_iterations=20)
    first = core._invert(forward, np.log(observed[:3]), np.log(initial[:, :3]), None, short)
    np.savez_compressed(
        os.environ["GOLDEN_TARGET"],
        first_iteration_models=np.asarray(first.log_models).T.copy(),
        first_iteration_chi2=np.asarray(first.chi2, dtype=float),
        observed_log=np.log(observed),
        initial_log=np.log(initial).T.copy(),
        final_log_models=np.asarray(result.final_log_models).T.copy(),
        predicted_log=np.asarray(result.predicted_log_data),
        window_final_chi2=np.asarray([r["final_chi2_data"] for r in result.window_reports], dtype=float),
        window_iterations=np.asarray([r["iterations"] for r in result.window_reports]),
        settings=np.asarray([ITERATIONS, DATA_STD, 50.0, 10.0]),
    )


def main() -> None:
    if len(sys.argv) == 2 and sys.argv[1] == "--child":
        _child()
        return
    if not (REFERENCE / "adtlert").is_dir():
        raise SystemExit("set ADTLERT_REFERENCE to the AD-TLERT project root (the folder holding adtlert/)")
    from make_golden import _stub_meshio

    with tempfile.TemporaryDirectory() as stub:
        _stub_meshio(Path(stub))
        env = dict(os.environ, PYTHONPATH=os.pathsep.join((stub, str(REFERENCE), str(HERE))),
                   ADTLERT_ENABLE_FLOAT64="1", GOLDEN_TARGET=str(TARGET), OMP_NUM_THREADS="1")
        subprocess.run([sys.executable, __file__, "--child"], check=True, env=env)
    print("wrote", TARGET.name, f"{TARGET.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
