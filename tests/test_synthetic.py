"""CPU checks of the seeded benchmark workloads: sizes, surveys and model statistics."""

import numpy as np

from adtlert_b200 import Mesh, Mesh3D, Survey, synthetic
from adtlert_b200.fem import inverse_cosine_weights, wavenumber_bounds


def test_flat_section_sizes():
    nodes, cells, electrodes, rows = synthetic.flat_section()
    assert (len(nodes), len(cells), len(electrodes), len(rows)) == (4961, 9600, 48, 1232)
    assert len(synthetic.flat_section(3)[3]) == 612


def test_terrain_section():
    nodes, cells, surface, electrodes, rows = synthetic.terrain_section()
    assert (len(cells), len(electrodes), len(rows)) == (40000, 96, 2538)
    mesh = Mesh.from_arrays(nodes, cells, surface_node_ids=surface)
    assert mesh.cell_count == 40000
    # surface and sides unjittered: electrodes sit on surface nodes at 1 m spacing
    assert np.allclose(np.diff(electrodes[:, 0]), 1.0)
    assert np.allclose(nodes[surface, 0], np.arange(201))
    # interior columns jittered by at most 0.05 m, and not all in line
    offsets = nodes[:, 0] - np.rint(nodes[:, 0])
    assert np.abs(offsets).max() <= 0.05 + 1e-12 and np.abs(offsets).max() > 0.01
    # every triangle counter-clockwise with positive area
    p = nodes[cells]
    area = 0.5 * ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    assert area.min() > 0
    # |surface| <= 5 m, depth 50 m
    assert np.abs(nodes[surface, 1]).max() <= 5.0
    assert np.isclose((nodes[surface, 1] - nodes[surface + 100 * 201, 1]).mean(), 50.0)
    # distinct ABMN rows, four distinct electrodes each; 19 wavenumbers (r_min 0.5 m, r_max 190 m)
    assert len({tuple(r) for r in rows.tolist()}) == len(rows)
    assert all(len(set(r)) == 4 for r in rows.tolist())
    assert len(inverse_cosine_weights(*wavenumber_bounds(electrodes))[0]) == 19
    Survey.from_arrays(electrodes, rows)


def test_correlated_model_statistics():
    nodes, cells, *_ = synthetic.terrain_section()
    a, b = synthetic.correlated_model(nodes, cells, 0), synthetic.correlated_model(nodes, cells, 1)
    assert a.dtype == np.float32 and np.all(a > 0)
    log_rho = np.log10(1.0 / a.astype(float))
    assert abs(log_rho.mean() - 2.0) < 0.1 and abs(log_rho.std() - 0.4) < 0.05
    assert not np.array_equal(a, b)
    assert np.array_equal(a, synthetic.correlated_model(nodes, cells, 0))  # seeded
    # correlated: neighbouring cells (the two triangles of a quad) are close in log resistivity
    pairs = np.log10(1.0 / a.astype(float)).reshape(-1, 2)
    assert np.abs(pairs[:, 0] - pairs[:, 1]).mean() < 0.2 * log_rho.std()


def test_box_section_and_grid_survey():
    nodes, cells = synthetic.box_section()
    assert (len(nodes), len(cells)) == (45018, 244800)
    mesh = Mesh3D.from_arrays(nodes, cells)
    assert mesh.cell_count == 244800
    electrodes, rows = synthetic.grid_survey()
    assert electrodes.shape == (96, 3) and len(rows) == 4000
    assert len({tuple(r) for r in rows.tolist()}) == 4000
    # every current and potential dipole joins grid neighbours 4 m apart
    for pair in (rows[:, :2], rows[:, 2:]):
        a, b = pair.T
        assert np.allclose(np.linalg.norm(electrodes[a] - electrodes[b], axis=1), 4.0)
    assert all(len(set(r)) == 4 for r in rows.tolist())


def test_ellipsoid_model():
    nodes, cells = synthetic.box_section(30, 20, 10)
    sigma = synthetic.ellipsoid_model(nodes, cells, 0)
    rho = 1.0 / sigma.astype(float)
    assert sigma.dtype == np.float32
    values, counts = np.unique(np.round(rho, 3), return_counts=True)
    assert values[np.argmax(counts)] == 100.0  # background
    assert rho.min() >= 10.0 - 1e-3 and rho.max() <= 1000.0 + 1e-2
    assert len(values) >= 2
