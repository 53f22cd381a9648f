"""The terrain CPU baseline (the bench's reference-path restatement, TEST INFRASTRUCTURE) is
pinned to the reference's own terrain Jacobians: fields by SciPy SuperLU on the refined field
discretization, unit potentials solved on the quadratic auxiliary discretization, the C
contraction, refined cells summed into model cells."""

import numpy as np
import pytest

from adtlert_b200.discretization import build_discretization, exact_node_indices
from adtlert_b200.ert2p5d import space_problem
from adtlert_b200.fem import inverse_cosine_weights, wavenumber_bounds
from adtlert_b200.geometry import Mesh, Survey
from cases import case_inputs
from conftest import ROOT, assert_close
from oracle import baseline


@pytest.mark.parametrize("name", ["tri_terrain", "quad_terrain"])
def test_terrain_baseline_matches_the_reference(name):
    inputs = case_inputs(name)
    mesh = Mesh.from_arrays(inputs["nodes"], inputs["cells"], surface_node_ids=inputs["surface_node_ids"])
    survey = Survey.from_arrays(inputs["electrodes"], inputs["measurements"])
    k, w = inverse_cosine_weights(*wavenumber_bounds(survey.electrode_positions))

    def build(kind, **options):
        return build_discretization(kind, mesh, survey, k, auxiliary=True, refine=True, quadrature_order=2, **options)

    fields_space, potential_space = build("primary"), build("primary_potential", quadratic=True)
    primary = baseline.unit_potentials(space_problem(potential_space, mesh, survey, k, w))
    primary = primary[..., exact_node_indices(potential_space.dof_nodes, fields_space.dof_nodes)]
    oracle = baseline.TerrainBaseline(space_problem(fields_space, mesh, survey, k, w), primary)
    fields = oracle.fields(np.asarray(inputs["sigma"], dtype=np.float64))
    J = oracle.jacobian_rows(fields, np.arange(len(inputs["measurements"])), threads=2)
    golden = np.load(ROOT / "tests" / "golden" / f"{name}_float64.npz")
    assert_close(J, golden["jacobian"], 1e-8, f"{name}: CPU baseline Jacobian vs the reference (float64)")
