"""The FP64 oracle of the windowed Gauss-Newton inversion against AD-TLERT's own driver.

``tests/golden/timelapse_small.npz`` holds the reference's ``invert_windowed_timelapse_log_
resistivity`` run in float64 on a small seeded series, and one Gauss-Newton iteration of its first
window with a 20-iteration CGLS (``make_timelapse_golden.py``).

CGLS truncated at the example's 60 iterations is sensitive to rounding on these systems: given
the reference's own matrix the oracle's CGLS reproduces the reference's step exactly, but a
1e-13 perturbation of the matrix (two FP64 Jacobians that differ only in summation order) moves
the 60-iteration step by ~2e-2, and the final models of a 4-iteration window by ~2e-4. So the
linearized system and step are pinned tightly through the 20-iteration case, where no such
amplification occurs, and the full run at the algorithm's own sensitivity."""

import numpy as np

from cases import case_inputs
from conftest import ROOT, assert_close
from oracle.timelapse import OracleTimeLapse


def _oracle(golden, **overrides):
    iterations, data_std, regularization, temporal = golden["settings"]
    inputs = case_inputs("tri_flat")
    options = dict(max_iterations=int(iterations), data_std=data_std, regularization=regularization,
                   temporal_regularization=temporal)
    options.update(overrides)
    return OracleTimeLapse(inputs["nodes"], inputs["cells"], inputs["electrodes"], inputs["measurements"], **options)


def test_one_iteration_matches_the_reference_tightly():
    golden = np.load(ROOT / "tests" / "golden" / "timelapse_small.npz")
    oracle = _oracle(golden, max_iterations=1, cgls_max_iterations=20)
    models, _, chi2, _ = oracle.invert_window(golden["observed_log"][:3], golden["initial_log"][:3])
    assert_close(models, golden["first_iteration_models"], 1e-9, "models after one iteration")
    assert_close(chi2, golden["first_iteration_chi2"], 1e-9, "chi2 after one iteration")


def test_windowed_run_matches_the_reference():
    golden = np.load(ROOT / "tests" / "golden" / "timelapse_small.npz")
    oracle = _oracle(golden)
    final, histories = oracle.run(golden["observed_log"], golden["initial_log"])
    assert_close(final, golden["final_log_models"], 1e-3, "final log models")
    assert [len(h) for h in histories] == list(golden["window_iterations"])
    assert_close([h[-1] for h in histories], golden["window_final_chi2"], 2e-3, "window chi2")
    predicted = np.stack([oracle.linearize(row)[0] for row in final])
    assert_close(predicted, golden["predicted_log"], 1e-4, "predicted log data")
