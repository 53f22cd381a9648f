"""3D P1/P2 tetrahedral DC operator on the B200 kernels of ``libadtlert_b200``.

Drop-in for ``adtlert.forward.ERTForward3D`` (adtlert/forward/ert3d.py:114-983): same
constructor options, methods, keyword arguments, exceptions and CPU results. One model is one
symmetric positive definite system (a single wavenumber 0 of weight 1 in the plan). Its field
columns are

* singularity removal on a flat surface: one column per current electrode with the right-hand
  side A(1) u_p (u_p = (1/r + 1/r') / 4 pi, the half-space primary potential), followed by one
  column per receiver electrode with its point-source interpolation row;
* otherwise: one point-source column per electrode used as current or receiver, shared by both
  roles (the reference's ``_shared_source_receiver_rhs``, ert3d.py:212-218, generalised).

Resistances gather current columns at receiver electrodes; the Jacobian is the electrode Gram of
the current and receiver columns; vjp/jvp are the same Gram contractions with the Robin terms, so
no adjoint or tangent solve is needed (the operator is symmetric: the receiver columns are the
adjoint fields of unit measurement cotangents).
"""

from __future__ import annotations

import contextlib
import ctypes
import hashlib
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from . import tuning as _tuning
from .graph import JacobianGraph
from .ert2p5d import _checked_to_host, _Slots, _survey_arrays
from .field_store import FieldStore, model_fingerprints
from .geometry3d import (
    Mesh3D,
    p2_shape_values,
    p2_triangle_mass,
    quadratic_topology,
    tetrahedron_p2_stiffness,
    tetrahedron_stiffness,
)
from .inputs import (
    FLOAT_DTYPE,
    cell_vector,
    check_finite,
    conductivity_model,
    conductivity_series,
    cotangent_series,
    measurement_vector,
    option,
    parameter_targets,
)

Tensor = torch.Tensor

ELECTRODE_RADIUS_FRACTION = 0.5  # fallback radius of a source on a node (ert3d.py:47)
MAX_COLUMNS = 200  # field columns per model (kMaxColumns of the library)
FACE_MASS = np.asarray(((2.0, 1.0, 1.0), (1.0, 2.0, 1.0), (1.0, 1.0, 2.0))) / 12.0


@dataclass(frozen=True)
class ForwardResponse3D:
    """Result of a 3D DC solve; the potentials are ``None`` unless requested (CPU tensors)."""

    apparent_resistivity: Tensor
    resistance: Tensor
    electrode_potentials: Tensor | None = None
    node_potentials: Tensor | None = None


@dataclass
class Problem3D:
    """Host arrays of one 3D plan (what ``adt_plan_create`` copies) and its right-hand sides."""

    arrays: dict
    counts: dict
    current_ids: np.ndarray
    receiver_ids: np.ndarray
    columns: list
    current_columns: np.ndarray
    receiver_columns: np.ndarray
    electrode_matrix: np.ndarray
    fixed: np.ndarray
    unit_primary: np.ndarray | None
    direct: np.ndarray | None

    def struct(self) -> _native.Problem:
        a, c = self.arrays, self.counts
        h = _native.host_ptr
        K, BL = a["cell_dofs"].shape[1], a["bdofs"].shape[1]
        return _native.Problem(
            dof_count=c["N"], dim=3, dof_coordinates=h(a["coords"]), cell_count=c["C"], local_dofs=K,
            cell_dofs=h(a["cell_dofs"]), stiffness=h(a["stiffness"]), mass=h(a["mass"]), parent_cells=None,
            model_cell_count=c["C"], boundary_count=c["Nb"], boundary_local=BL, boundary_dofs=h(a["bdofs"]),
            boundary_cells=h(a["bcells"]), boundary_mass=h(a["bmass"]), boundary_coefficients=h(a["bcoef"]),
            wavenumber_count=1, wavenumbers=h(a["k"]), weights=h(a["w"]), electrode_count=c["E"],
            receiver_width=K, receiver_dofs=h(a["rdofs"]), receiver_weights=h(a["rw"]),
            measurement_count=c["D"], abmn=h(a["abmn"]), source_cell_ptr=h(a["sptr"]), source_cells=h(a["scells"]),
            fixed_count=len(self.fixed), fixed_dofs=h(a["fixed"]) if len(self.fixed) else None,
        )


def electrode_rows(slots: np.ndarray, electrode_count: int) -> np.ndarray:
    """Electrodes used in ``slots`` (remote slot excluded), ascending (ert3d.py:93-106)."""

    ids = np.unique(slots)
    return ids[ids < electrode_count].astype(np.int64)


def primary_potential(nodes: np.ndarray, source: np.ndarray, surface_z: float) -> np.ndarray:
    """Unit half-space potential (1/r + 1/r')/(4 pi) of a point source and its image above the
    surface level; distances at or below 1e-12 take half the nearest node distance
    (ert3d.py:367-385)."""

    mirror = np.array(source, dtype=float)
    mirror[2] = 2.0 * surface_z - source[2]
    direct = np.linalg.norm(nodes - source, axis=1)
    image = np.linalg.norm(nodes - mirror, axis=1)
    fallback = max(float(np.min(direct[direct > 1e-12])) * ELECTRODE_RADIUS_FRACTION, 1e-12)
    direct = np.where(direct > 1e-12, direct, fallback)
    image = np.where(image > 1e-12, image, fallback)
    return (1.0 / direct + 1.0 / image) / (4.0 * np.pi)


def robin_faces(mesh: Mesh3D, center: np.ndarray, face_dofs: np.ndarray, element_order: int = 1):
    """Far-field faces (their dofs: 3 for P1, 6 for P2) with their Robin boundary mass alpha *
    M_face (area * the linear face mass, or the quadratic one), alpha = max(r.n / |r|^2, 0) for r
    from the electrode centroid to the face center; surface faces and faces with alpha = 0 carry
    none (ert3d.py:224-256)."""

    width = face_dofs.shape[1]
    faces, cells, masses = [], [], []
    for f in np.flatnonzero(~mesh.surface_face_mask):
        radial = mesh.boundary_face_centers[f] - center
        r2 = float(radial @ radial)
        if r2 <= 0.0:
            continue
        alpha = max(float(radial @ mesh.boundary_face_normals[f]) / r2, 0.0)
        if alpha == 0.0:
            continue
        faces.append(face_dofs[f])
        cells.append(mesh.boundary_face_cells[f])
        area = mesh.boundary_face_areas[f]
        masses.append(alpha * (p2_triangle_mass(area) if element_order == 2 else area * FACE_MASS))
    if not faces:
        return np.zeros((0, width), np.int32), np.zeros(0, np.int32), np.zeros((0, width, width))
    return np.asarray(faces, np.int32), np.asarray(cells, np.int32), np.asarray(masses)


def build_problem_3d(mesh: Mesh3D, survey, boundary_mode: str = "mixed",
                     singularity_removal: bool = True, element_order: int = 1) -> Problem3D:
    """Templates, Robin faces, Dirichlet dofs, field columns and right-hand sides of a P1 or
    ten-node P2 operator (ert3d.py:140-413), built on the host without a GPU. P2 dofs are the
    vertices and the edge midpoints (quadratic_topology); electrodes interpolate with the P2
    shape functions at their barycentric coordinates (ert3d.py:71-90)."""

    if element_order == 2:
        nodes, cells, face_dofs = quadratic_topology(mesh.nodes, mesh.cells, mesh.boundary_faces)
        stiffness = tetrahedron_p2_stiffness(mesh.nodes, mesh.cells)
    else:
        nodes, cells, face_dofs = mesh.nodes, mesh.cells, mesh.boundary_faces
        stiffness = tetrahedron_stiffness(mesh.nodes, mesh.cells)
    K = cells.shape[1]
    N, C, E = len(nodes), mesh.cell_count, survey.electrode_count
    positions = np.asarray(survey.electrode_positions, dtype=float)
    slots = survey.measurement_slots()
    current_ids = electrode_rows(slots[:, :2], E)
    receiver_ids = electrode_rows(slots[:, 2:], E)
    singular = bool(singularity_removal and mesh.is_flat_surface)
    if singular:
        columns = [("primary", int(e)) for e in current_ids] + [("point", int(e)) for e in receiver_ids]
        current_col = {int(e): i for i, e in enumerate(current_ids)}
        receiver_col = {int(e): len(current_ids) + i for i, e in enumerate(receiver_ids)}
    else:
        union = np.union1d(current_ids, receiver_ids)
        columns = [("point", int(e)) for e in union]
        current_col = receiver_col = {int(e): i for i, e in enumerate(union)}
    Ec = len(columns)
    if Ec > MAX_COLUMNS:
        raise ValueError(f"{Ec} field columns exceed the {MAX_COLUMNS} supported by the sensitivity kernels")
    cell_ids, bary = mesh.locate_points(positions)
    weights = p2_shape_values(bary) if element_order == 2 else bary
    electrode_matrix = np.zeros((E, N))
    np.add.at(electrode_matrix, (np.repeat(np.arange(E), K), cells[cell_ids].reshape(-1)), weights.reshape(-1))

    def mapped(role: dict, values: np.ndarray) -> np.ndarray:
        return np.asarray([Ec if v == E else role[int(v)] for v in values], dtype=np.int32)

    abmn = np.stack((mapped(current_col, slots[:, 0]), mapped(current_col, slots[:, 1]),
                     mapped(receiver_col, slots[:, 2]), mapped(receiver_col, slots[:, 3])), axis=1)
    electrodes = np.asarray([e for _, e in columns], dtype=np.int64)
    unit_primary = direct = None
    if singular:
        unit_primary = np.zeros((1, Ec, N))
        for i, (kind, e) in enumerate(columns):
            if kind == "primary":
                unit_primary[0, i] = primary_potential(nodes, positions[e], mesh.surface_reference_level)
    points = [i for i, (kind, _) in enumerate(columns) if kind == "point"]
    if points:
        direct = np.zeros((1, Ec, N))
        direct[0, points] = electrode_matrix[electrodes[points]]
    BL = face_dofs.shape[1]
    if boundary_mode == "mixed":
        bdofs, bcells, bmass = robin_faces(mesh, positions.mean(axis=0), face_dofs, element_order)
        fixed = np.zeros(0, dtype=np.int32)
    else:
        bdofs, bcells, bmass = np.zeros((0, BL), np.int32), np.zeros(0, np.int32), np.zeros((0, BL, BL))
        fixed = np.unique(face_dofs[~mesh.surface_face_mask].reshape(-1)).astype(np.int32)
    arrays = {
        "coords": np.ascontiguousarray(nodes, dtype=np.float64),
        "cell_dofs": np.ascontiguousarray(cells, dtype=np.int32),
        "stiffness": np.ascontiguousarray(stiffness, dtype=np.float64),
        "mass": np.zeros((C, K, K)),
        "bdofs": np.ascontiguousarray(bdofs, dtype=np.int32),
        "bcells": np.ascontiguousarray(bcells, dtype=np.int32),
        "bmass": np.ascontiguousarray(bmass, dtype=np.float64),
        "bcoef": np.ones((1, len(bdofs))),
        "k": np.zeros(1),
        "w": np.ones(1),
        "rdofs": np.ascontiguousarray(cells[cell_ids[electrodes]], dtype=np.int32),
        "rw": np.ascontiguousarray(weights[electrodes], dtype=np.float64),
        "abmn": np.ascontiguousarray(abmn, dtype=np.int32),
        "sptr": np.zeros(Ec + 1, dtype=np.int32),
        "scells": np.zeros(1, dtype=np.int32),
        "fixed": np.ascontiguousarray(fixed, dtype=np.int32),
    }
    counts = {"N": N, "C": C, "Nb": len(bdofs), "E": Ec, "D": survey.measurement_count}
    return Problem3D(
        arrays, counts, current_ids, receiver_ids, columns,
        np.asarray([current_col[int(e)] for e in current_ids], dtype=np.int64),
        np.asarray([receiver_col[int(e)] for e in receiver_ids], dtype=np.int64),
        electrode_matrix, fixed,
        None if unit_primary is None else np.ascontiguousarray(unit_primary),
        None if direct is None else np.ascontiguousarray(direct),
    )


def _mesh3d(mesh) -> Mesh3D:
    """Our Mesh3D for the reference's or our own mesh object (the surface mask is kept)."""

    if isinstance(mesh, Mesh3D):
        return mesh
    mask = getattr(mesh, "surface_face_mask", None)
    faces = getattr(mesh, "boundary_faces", None)
    ours = Mesh3D.from_arrays(np.asarray(mesh.nodes, dtype=float), np.asarray(mesh.cells))
    if mask is None or faces is None:
        return ours
    # carry the caller's surface choice over by face (face rows are sorted the same way)
    if np.array_equal(np.asarray(faces), ours.boundary_faces):
        return Mesh3D.from_arrays(ours.nodes, ours.cells, surface_face_mask=np.asarray(mask, dtype=bool))
    return ours


class ERTForward3D:
    """3D tetrahedral DC operator (P1 or ten-node P2, mixed or Dirichlet far field) on B200 kernels."""

    def __init__(self, mesh, survey, boundary_mode: str = "mixed", singularity_removal: bool = True,
                 element_order: int = 1, geometric_factor_mode: str = "auto",
                 normal_field_cache_max_entries: int = 8, series_batch_steps: int = 1) -> None:
        self.boundary_mode = option(boundary_mode, ("mixed", "dirichlet"), "boundary_mode")
        self.geometric_factor_mode = option(geometric_factor_mode, ("auto", "analytic", "numerical"),
                                            "geometric_factor_mode")
        if not torch.cuda.is_available():
            raise RuntimeError("ADTLERT requires an NVIDIA GPU with CUDA (B200 kernels)")
        if element_order not in (1, 2):
            raise ValueError("element_order must be 1 or 2")
        self.source_mesh, self.source_survey = mesh, survey
        self.mesh = _mesh3d(mesh)
        self.survey = _survey_arrays(survey)
        if self.survey.dimension != 3:
            raise ValueError("ERTForward3D requires three-coordinate electrode positions")
        if int(series_batch_steps) < 1:
            raise ValueError("series_batch_steps must be >= 1")
        self.singularity_removal = bool(singularity_removal)
        self.element_order = int(element_order)
        self.series_batch_steps = int(series_batch_steps)
        self._field_cache = FieldStore(normal_field_cache_max_entries, self._fingerprints)
        self.normal_field_cache_max_entries = self._field_cache.capacity
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = _native.load_library()
        self._cache: dict = {}
        self._solver = _Slots()
        self._plan = None
        self._build()

    @classmethod
    def from_mesh_survey(cls, mesh, survey, **options) -> ERTForward3D:
        return cls(mesh, survey, **options)

    # ------------------------------------------------------------------ set-up
    def _build(self) -> None:
        problem = build_problem_3d(self.mesh, self.survey, self.boundary_mode, self.singularity_removal,
                                   self.element_order)
        self._problem = problem
        struct = problem.struct()
        plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _native.check(self._lib.adt_plan_create(ctypes.byref(struct), ctypes.byref(plan)), None, "adt_plan_create")
        self._plan = plan
        info = _native.PlanInfo()
        self._lib.adt_plan_get_info(plan, ctypes.byref(info))
        self.plan_info = {name: getattr(info, name) for name, _ in _native.PlanInfo._fields_}
        with torch.cuda.device(self.device):
            _native.check(
                self._lib.adt_set_static_rhs(plan, _native.host_ptr(problem.unit_primary),
                                             _native.host_ptr(problem.direct), self._stream()),
                plan, "adt_set_static_rhs")
        self.C, self.N = self.mesh.cell_count, problem.counts["N"]  # dofs (vertices + P2 midpoints)
        self.E, self.D = self.survey.electrode_count, self.survey.measurement_count
        self.columns = problem.counts["E"]
        self._current_electrode_ids = problem.current_ids
        self._receiver_electrode_ids = problem.receiver_ids

    @property
    def cell_count(self) -> int:
        return self.C

    def _stream(self):
        return _native.stream_handle(self.device)

    def kernel_launches(self) -> int:
        return int(self._lib.adt_kernel_launches(self._plan))

    def autotune(self, conductivity=None, *, repeats: int = 3, jacobian: bool = True) -> dict:
        """Choose the plan's launch shapes (solver strips, tiled split depth, Jacobian kernel) by
        timing them on ``conductivity``; returns the choice and its times (ms)."""

        return _tuning.autotune(self, conductivity, repeats, jacobian)

    def tuning(self) -> dict:
        return _tuning.tuning(self)

    def jacobian_graph(self) -> "JacobianGraph":
        """A CUDA graph of the whole fresh-model ``jacobian()`` chain, replayed per model."""

        return JacobianGraph(self)

    def set_tuning(self, settings: dict) -> None:
        _tuning.set_tuning(self, settings)

    def _call(self, name: str, *args) -> None:
        _native.check(getattr(self._lib, name)(self._plan, *args), self._plan, name)

    def _sigma(self, conductivity) -> Tensor:
        return conductivity_model(conductivity, self.C, torch.float64)

    def _series(self, conductivities) -> Tensor:
        return conductivity_series(conductivities, self.C, torch.float64)

    # ------------------------------------------------------------------ fields
    def _solve_fields(self, sigmas: Tensor, name) -> list[Tensor]:
        batch = int(sigmas.shape[0])
        sig = sigmas.to(self.device, torch.float32).contiguous()
        entry = self._solver.lookup(batch)
        self._call("adt_factorize", entry["slot"], _native.ptr(sig), batch, self._stream())
        entry["name"] = name
        self._solver.factorizations += 1
        fields = torch.empty((batch, 1, self.N, self.columns), dtype=torch.float32, device=self.device)
        self._call("adt_solve_fields", entry["slot"], _native.ptr(sig), batch, _native.ptr(fields), self._stream())
        check_finite(fields, "node fields")
        return [fields[i] for i in range(batch)]

    def _fingerprints(self, models: Tensor) -> list[bytes]:
        return model_fingerprints(self._lib, self._plan, models, self._stream())

    def _fields_series(self, models: Tensor):
        return self._field_cache.fields(models, self.series_batch_steps, self._solve_fields)

    def _fields(self, conductivity) -> Tensor:
        return self._fields_series(self._sigma(conductivity)[None])[0][0]

    def normal_field_cache_info(self) -> dict[str, int]:
        return self._field_cache.info()

    def _stack(self, fields: list[Tensor]) -> Tensor:
        if len(fields) == 1:
            return fields[0][None]
        return torch.stack(fields).contiguous()

    def _resistances(self, stacked: Tensor) -> Tensor:
        """Transfer resistances (S, D) float64 on the device of stacked fields (S, 1, N, E')."""

        S = int(stacked.shape[0])
        normal = torch.empty((S, self.D), dtype=torch.float64, device=self.device)
        reciprocal = torch.empty_like(normal)
        self._call("adt_measure", _native.ptr(stacked), S, _native.ptr(normal), _native.ptr(reciprocal),
                   None, self._stream())
        return normal

    # ------------------------------------------------------------------ forward API
    def _geometric_factors(self) -> Tensor:
        numerical = self.geometric_factor_mode == "numerical" or (
            self.geometric_factor_mode == "auto" and not self.mesh.is_flat_surface)
        if not numerical:
            return self._analytic_factors()
        if "geometric_factors" not in self._cache:
            ones = torch.ones((1, self.C), dtype=torch.float64)
            (fields,) = self._solve_fields(ones, None)
            unit = self._resistances(fields[None])[0]
            if bool(torch.any(torch.abs(unit) <= torch.finfo(torch.float64).tiny)):
                raise ValueError("numerical geometric-factor solve produced zero resistance")
            self._cache["geometric_factors"] = (1.0 / unit).cpu().to(FLOAT_DTYPE)
        return self._cache["geometric_factors"]

    def _analytic_factors(self) -> Tensor:
        if "analytic_factors" not in self._cache:
            self._cache["analytic_factors"] = torch.as_tensor(self.survey.geometric_factors(), dtype=FLOAT_DTYPE)
        return self._cache["analytic_factors"]

    def _per_electrode(self, rows: np.ndarray) -> Tensor:
        full = np.full((self.E, rows.shape[1]), np.nan)
        full[self._current_electrode_ids] = rows
        return torch.as_tensor(full, dtype=FLOAT_DTYPE)

    def _response(self, fields: Tensor, currents, include_fields: bool) -> ForwardResponse3D:
        resistance = self._resistances(fields[None])[0].cpu().to(FLOAT_DTYPE)
        apparent = self._geometric_factors() * resistance / torch.as_tensor(currents, dtype=FLOAT_DTYPE)
        if not include_fields:
            return ForwardResponse3D(apparent, resistance)
        nodes = torch.empty((self.columns, self.N), dtype=torch.float32, device=self.device)
        self._call("adt_integrated_potentials", _native.ptr(fields), _native.ptr(nodes), self._stream())
        current = nodes[torch.as_tensor(self._problem.current_columns, device=self.device)].cpu().numpy().astype(float)
        return ForwardResponse3D(
            apparent,
            resistance,
            electrode_potentials=self._per_electrode(current @ self._problem.electrode_matrix.T),
            node_potentials=self._per_electrode(current),
        )

    def solve(self, conductivity, currents=1.0) -> ForwardResponse3D:
        return self._response(self._fields(conductivity), currents, include_fields=True)

    def resistance(self, conductivity) -> Tensor:
        return self.resistance_series(self._sigma(conductivity)[None])[0]

    def resistance_series(self, conductivities) -> Tensor:
        resistance = self._resistances_device(self._series(conductivities)).cpu()
        check_finite(resistance, "resistances")
        return resistance

    def _resistances_device(self, models: Tensor) -> Tensor:
        """Resistances (S, D) of validated models (S, C), left on the GPU in the result dtype."""

        fields, _ = self._fields_series(models)
        return self._resistances(self._stack(fields)).to(FLOAT_DTYPE)

    def apparent_resistivity_values(self, conductivity, currents=1.0) -> Tensor:
        factors = self._geometric_factors()
        return factors * self.resistance(conductivity) / torch.as_tensor(currents, dtype=FLOAT_DTYPE)

    def apparent_resistivity_series(self, conductivities, currents=1.0) -> Tensor:
        factors = self._geometric_factors()
        resistance = self.resistance_series(conductivities)
        current = torch.as_tensor(currents, dtype=FLOAT_DTYPE)
        if current.ndim == 1 and current.shape[0] == resistance.shape[0] and current.shape[0] != resistance.shape[1]:
            current = current[:, None]
        return factors * resistance / current

    # ------------------------------------------------------------------ derivatives
    def _columns(self, cell_parameter_ids=None, parameter_count=None):
        ids, count = parameter_targets(cell_parameter_ids, parameter_count, self.C)
        if cell_parameter_ids is None:
            return None
        digest = hashlib.blake2b(ids.tobytes(), digest_size=16).digest()
        key = ("columns", digest, count)
        if key not in self._cache:
            active = np.flatnonzero(ids >= 0)
            order = active[np.argsort(ids[active], kind="stable")]
            ptr = np.concatenate(([0], np.cumsum(np.bincount(ids[active], minlength=count)))).astype(np.int32)
            self._cache[key] = (len(self._cache) + 1, count, ptr, np.ascontiguousarray(order, dtype=np.int32))
        return self._cache[key]

    def _aggregate(self, values: Tensor, columns) -> Tensor:
        if columns is None:
            return values
        key, count, ptr, cells = columns
        rows = int(values.shape[0])
        out = torch.empty((rows, count), dtype=torch.float32, device=self.device)
        self._call("adt_aggregate_columns", key, count, _native.host_ptr(ptr), _native.host_ptr(cells),
                   _native.ptr(values.contiguous()), rows, int(values.shape[1]), _native.ptr(out), self._stream())
        return out

    def _cell_products(self, fields: Tensor, cotangent: Tensor, robin: bool) -> Tensor:
        grad = torch.empty((1, self.C), dtype=torch.float32, device=self.device)
        self._call("adt_normal_vjp", _native.ptr(fields), _native.ptr(cotangent), int(robin), _native.ptr(grad),
                   self._stream())
        return grad

    def _data_products(self, fields: Tensor, direction: Tensor, robin: bool) -> Tensor:
        out = torch.empty(self.D, dtype=torch.float64, device=self.device)
        self._call("adt_normal_jvp", _native.ptr(fields), _native.ptr(direction), int(robin), _native.ptr(out),
                   self._stream())
        return out

    def vjp(self, conductivity, cotangent) -> Tensor:
        cotangent = measurement_vector(cotangent, self.D, FLOAT_DTYPE)
        return self.vjp_series(self._sigma(conductivity)[None], cotangent[None])[0]

    def vjp_series(self, conductivities, cotangents) -> Tensor:
        """Transposed exact resistance Jacobian applied to every step (Robin terms included)."""

        models = self._series(conductivities)
        cotangents = cotangent_series(cotangents, models.shape[0], self.D)
        gradient = self._vjp_device(models, cotangents).cpu()
        check_finite(gradient, "conductivity gradient")
        return gradient

    def _vjp_device(self, models: Tensor, cotangents: Tensor) -> Tensor:
        """Exact VJPs (S, C) float32 on the GPU of validated models and cotangents (S, D)."""

        fields, _ = self._fields_series(models)
        rows = [self._cell_products(f, c.to(self.device, torch.float64).contiguous(), True)[0]
                for f, c in zip(fields, cotangents, strict=True)]
        return torch.stack(rows)

    def jvp(self, conductivity, delta_conductivity) -> Tensor:
        result = self._jvp_device(self._sigma(conductivity), cell_vector(delta_conductivity, self.C, torch.float64))
        result = result.cpu().to(FLOAT_DTYPE)
        check_finite(result, "resistance jvp")
        return result

    def _jvp_device(self, sigma: Tensor, direction: Tensor) -> Tensor:
        """Resistance tangent (D,) float64 on the GPU of a validated model and direction (C,)."""

        fields = self._fields(sigma)
        return self._data_products(fields, direction.to(self.device, torch.float32).contiguous(), True)

    def normal_vjp(self, conductivity, cotangent, *, cell_parameter_ids=None, parameter_count=None) -> Tensor:
        cotangent = measurement_vector(cotangent, self.D, FLOAT_DTYPE)
        return self.normal_vjp_series(self._sigma(conductivity)[None], cotangent[None],
                                      cell_parameter_ids=cell_parameter_ids, parameter_count=parameter_count)[0]

    def normal_vjp_series(self, conductivities, cotangents, *, cell_parameter_ids=None,
                          parameter_count=None) -> Tensor:
        models = self._series(conductivities)
        cotangents = cotangent_series(cotangents, models.shape[0], self.D)
        columns = self._columns(cell_parameter_ids, parameter_count)
        fields, _ = self._fields_series(models)
        rows = [self._aggregate(self._cell_products(f, c.to(self.device, torch.float64).contiguous(), False),
                                columns)[0]
                for f, c in zip(fields, cotangents, strict=True)]
        gradient = torch.stack(rows).cpu()
        check_finite(gradient, "normal sensitivity vjp")
        return gradient

    def normal_jvp(self, conductivity, delta_conductivity) -> Tensor:
        fields = self._fields(conductivity)
        direction = cell_vector(delta_conductivity, self.C, torch.float64)
        result = self._data_products(fields, direction.to(self.device, torch.float32).contiguous(), False)
        result = result.cpu().to(FLOAT_DTYPE)
        check_finite(result, "normal sensitivity jvp")
        return result

    def _jacobian_device(self, fields: Tensor, include_robin: bool, columns) -> Tensor:
        J = torch.empty((self.D, self.C), dtype=torch.float32, device=self.device)
        self._call("adt_normal_jacobian", _native.ptr(fields), 0, self.D, _native.ptr(J), self._stream())
        if include_robin:
            self._call("adt_boundary_jacobian", _native.ptr(fields), 0, self.D, _native.ptr(J), self._stream())
        return self._aggregate(J, columns)

    def jacobian(self, conductivity, *, batch_size=None, include_robin_boundary_derivative: bool = False,
                 normal_sensitivity: bool = True, jacobian_cell_parameter_ids=None,
                 jacobian_parameter_count=None) -> Tensor:
        """Explicit resistance Jacobian ``-(u_M - u_N)_c^T T_c (u_A - u_B)_c`` (ert3d.py:867-927).

        Every row is computed in one launch; ``batch_size`` is validated as in the reference and
        does not change the result. 3D responses are not reciprocity-averaged, so
        ``normal_sensitivity`` has no effect.
        """

        del normal_sensitivity
        if batch_size is not None and int(batch_size) < 1:
            raise ValueError("batch_size must be >= 1")
        columns = self._columns(jacobian_cell_parameter_ids, jacobian_parameter_count)
        fields = self._fields(conductivity)
        return _checked_to_host(self._jacobian_device(fields, include_robin_boundary_derivative, columns), "jacobian")

    def jacobian_columnwise(self, conductivity) -> Tensor:
        basis = torch.eye(self.C, dtype=FLOAT_DTYPE)
        return torch.stack([self.jvp(conductivity, column) for column in basis], dim=1)

    def solve_with_jacobian(self, conductivity, currents=1.0, *, batch_size=None,
                            include_robin_boundary_derivative: bool = False, normal_sensitivity: bool = True,
                            include_fields: bool = False, jacobian_cell_parameter_ids=None,
                            jacobian_parameter_count=None):
        response, jacobian = self._solve_with_jacobian_device(
            conductivity, currents, batch_size=batch_size,
            include_robin_boundary_derivative=include_robin_boundary_derivative,
            normal_sensitivity=normal_sensitivity, include_fields=include_fields,
            jacobian_cell_parameter_ids=jacobian_cell_parameter_ids,
            jacobian_parameter_count=jacobian_parameter_count)
        return response, _checked_to_host(jacobian, "jacobian")

    def _solve_with_jacobian_device(self, conductivity, currents=1.0, *, batch_size=None,
                                    include_robin_boundary_derivative: bool = False, normal_sensitivity: bool = True,
                                    include_fields: bool = False, jacobian_cell_parameter_ids=None,
                                    jacobian_parameter_count=None):
        """The response (CPU) and the Jacobian still on the device (float32)."""

        del normal_sensitivity
        if batch_size is not None and int(batch_size) < 1:
            raise ValueError("batch_size must be >= 1")
        sigma = self._sigma(conductivity)
        fields = self._fields(sigma)
        response = self._response(fields, currents, include_fields=include_fields)
        columns = self._columns(jacobian_cell_parameter_ids, jacobian_parameter_count)
        return response, self._jacobian_device(fields, include_robin_boundary_derivative, columns)

    def prepare(self, conductivity=None, *, include_solver_state: bool = True) -> None:
        self._geometric_factors()
        if include_solver_state:
            self._fields(torch.ones(self.C, dtype=FLOAT_DTYPE) if conductivity is None else conductivity)

    # ------------------------------------------------------------------ lifetime
    def close(self) -> None:
        self._field_cache.clear()
        self._solver.close()

    def __del__(self) -> None:
        with contextlib.suppress(Exception):
            if self._plan is not None:
                torch.cuda.synchronize(self.device)
                self._lib.adt_plan_destroy(self._plan)
                self._plan = None


__all__ = ["ERTForward3D", "ForwardResponse3D", "Mesh3D", "build_problem_3d"]
