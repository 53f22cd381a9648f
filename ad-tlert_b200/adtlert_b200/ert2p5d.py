"""2.5D multi-wavenumber ERT operator on the B200 kernels of ``libadtlert_b200``.

Drop-in for ``adtlert.forward.ERTForward2p5D`` (adtlert/forward/ert2p5d.py:108-1121): same
constructor, methods, keyword arguments, defaults, exceptions and return devices (results on
the CPU). Every wavenumber is solved with the secondary-field formulation

    A(sigma) u_s = A(1) u_p - A(sigma) (rho_src u_p),    u = u_s + rho_src u_p,

with the analytic half-space primary field of each electrode on flat surfaces. On terrain the
fields live on an H2-refined auxiliary mesh and u_p is the numerical unit-conductivity potential
of a quadratic auxiliary discretization (solved once on the GPU, optionally cached on disk);
geometric factors may come from the same kind of solve. The host builds the element templates
and boundary terms once; assembly, the batched direct solves, quadrature, the ABMN gathers and
every derivative run as CUDA kernels on the caller's current stream.
"""

from __future__ import annotations

import contextlib
import ctypes
import hashlib
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import _native
from . import tuning as _tuning
from .graph import JacobianGraph
from .fem import (
    analytic_primary,
    boundary_mass,
    inverse_cosine_weights,
    quad_templates,
    robin_coefficients,
    triangle_templates,
    wavenumber_bounds,
)
from .discretization import Discretization, build_discretization, exact_node_indices
from .field_store import FieldStore, adjoint_batches, batch_name, model_fingerprints
from .geometry import Mesh, Survey, geometric_factors, locate_points
from .inputs import (
    FLOAT_DTYPE,
    cell_vector,
    check_finite,
    conductivity_model,
    finite_flag,
    conductivity_series,
    cotangent_series,
    measurement_vector,
    option,
    parameter_targets,
)

Tensor = torch.Tensor


@dataclass(frozen=True)
class ForwardResponse:
    """Result of a 2.5D ERT forward solve (CPU tensors)."""

    apparent_resistivity: Tensor
    resistance: Tensor
    electrode_potentials: Tensor
    integrated_potentials: Tensor
    wavenumbers: Tensor
    weights: Tensor


@dataclass
class _Fields:
    """Total fields (W, N, E) of one model on the GPU, dofs in the plan's solver order."""

    total: Tensor

    def on(self, device) -> Tensor:
        return self.total.to(device)


class _Slots:
    """Factor slots of the plan, keyed by batch size, each remembering which models it holds.

    Mirrors the naming contract of the reference's BatchedSolver (adtlert/forward/cudss.py:63-122):
    a slot is reused only when the requested factorization name equals the recorded one; any
    unnamed factorization forgets the record.
    """

    def __init__(self) -> None:
        self.slots: dict[int, dict] = {}
        self.factorizations = 0
        self._next = 0

    def lookup(self, models: int) -> dict:
        if models not in self.slots:
            self.slots[models] = {"slot": self._next, "name": None}
            self._next += 1
        return self.slots[models]

    def private(self) -> int:
        """A slot outside the batch-size table (a captured graph's): never reused by name."""

        self._next += 1
        return self._next - 1

    def holds(self, models: int, name) -> bool:
        entry = self.slots.get(models)
        return entry is not None and name is not None and entry["name"] == name

    def close(self) -> None:
        for entry in self.slots.values():
            entry["name"] = None


@dataclass
class ProblemArrays:
    """Host arrays of one 2.5D plan (what ``adt_plan_create`` copies), built without a GPU."""

    arrays: dict
    wavenumbers: np.ndarray
    weights: np.ndarray
    stiffness: np.ndarray
    mass: np.ndarray
    boundary_mass: np.ndarray
    robin: np.ndarray
    electrode_matrix: np.ndarray
    source_nodes: np.ndarray
    source_cells: np.ndarray
    counts: dict

    def struct(self) -> _native.Problem:
        a, c = self.arrays, self.counts
        h = _native.host_ptr
        return _native.Problem(
            dof_count=c["N"], dim=2, dof_coordinates=h(a["coords"]), cell_count=c["C"], local_dofs=c["K"],
            cell_dofs=h(a["cell_dofs"]), stiffness=h(a["stiffness"]), mass=h(a["mass"]),
            parent_cells=h(a.get("parents")), model_cell_count=c.get("Cm", c["C"]), boundary_count=c["Nb"],
            boundary_local=c.get("BL", 2), boundary_dofs=h(a["bdofs"]), boundary_cells=h(a["bcells"]),
            boundary_mass=h(a["bmass"]), boundary_coefficients=h(a["bcoef"]), wavenumber_count=c["W"],
            wavenumbers=h(a["k"]), weights=h(a["w"]), electrode_count=c["E"],
            receiver_width=c.get("RW", c["K"]), receiver_dofs=h(a["rdofs"]), receiver_weights=h(a["rw"]),
            measurement_count=c["D"], abmn=h(a["abmn"]), source_cell_ptr=h(a["sptr"]), source_cells=h(a["scells"]),
        )


def build_problem(mesh: Mesh, survey: Survey, quadrature_order: int = 2) -> ProblemArrays:
    """Quadrature, element templates, mixed-boundary coefficients, electrode interpolation and
    source-resistivity cells of a flat-surface operator (``build_discretization("native")``,
    adtlert/forward/discretization.py:485-575, and ert2p5d.py:158-216)."""

    positions = survey.electrode_positions[:, :2]
    k, w = inverse_cosine_weights(*wavenumber_bounds(survey.electrode_positions))
    nodes, cells = mesh.nodes, mesh.cells
    if cells.shape[1] == 3:
        stiffness, mass = triangle_templates(nodes, cells, quadrature_order)
    else:
        stiffness, mass = quad_templates(nodes, cells)
    bmass = boundary_mass(mesh.boundary_edge_lengths)
    robin = robin_coefficients(mesh.boundary_edge_centers, mesh.boundary_edge_normals, mesh.surface_edge_mask,
                               mesh.surface_reference_level, positions.mean(axis=0), k)
    cell_ids, interp = locate_points(nodes, cells, positions)
    E, N, K = survey.electrode_count, mesh.node_count, cells.shape[1]
    receiver_dofs = cells[cell_ids].astype(np.int32)
    electrode_matrix = np.zeros((E, N))
    np.add.at(electrode_matrix, (np.repeat(np.arange(E), K), receiver_dofs.reshape(-1)), interp.reshape(-1))
    distance = np.linalg.norm(nodes[None] - positions[:, None], axis=2)
    nearest = np.argmin(distance, axis=1)
    source_nodes = np.where(distance[np.arange(E), nearest] <= 1e-2, nearest, -1)
    ptr, lists = [0], []
    for e, node in enumerate(source_nodes):
        around = np.flatnonzero((cells == node).any(axis=1)) if node >= 0 else np.asarray([cell_ids[e]])
        lists.append(around)
        ptr.append(ptr[-1] + len(around))
    arrays = {
        "coords": np.ascontiguousarray(nodes, dtype=np.float64),
        "cell_dofs": np.ascontiguousarray(cells, dtype=np.int32),
        "stiffness": np.ascontiguousarray(stiffness, dtype=np.float64),
        "mass": np.ascontiguousarray(mass, dtype=np.float64),
        "bdofs": np.ascontiguousarray(mesh.boundary_edges, dtype=np.int32),
        "bcells": np.ascontiguousarray(mesh.boundary_edge_cells, dtype=np.int32),
        "bmass": np.ascontiguousarray(bmass, dtype=np.float64),
        "bcoef": np.ascontiguousarray(robin, dtype=np.float64),
        "k": np.ascontiguousarray(k, dtype=np.float64),
        "w": np.ascontiguousarray(w, dtype=np.float64),
        "rdofs": np.ascontiguousarray(receiver_dofs, dtype=np.int32),
        "rw": np.ascontiguousarray(interp, dtype=np.float64),
        "abmn": np.ascontiguousarray(survey.measurement_slots(), dtype=np.int32),
        "sptr": np.asarray(ptr, dtype=np.int32),
        "scells": np.ascontiguousarray(np.concatenate(lists), dtype=np.int32),
    }
    counts = {"N": N, "C": mesh.cell_count, "K": K, "Nb": len(mesh.boundary_edges), "W": len(k), "E": E,
              "D": survey.measurement_count}
    return ProblemArrays(arrays, k, w, stiffness, mass, bmass, robin, electrode_matrix, source_nodes, cell_ids, counts)


def source_cells(mesh: Mesh, survey: Survey):
    """Source node of every electrode (an input-mesh node within 1e-2, else -1) and the model
    cells whose conductivities set its source resistivity: the cells around that node, else the
    containing cell (ert2p5d.py:185-193, 480-511). Returns (nodes, containing cells, ptr, cells)."""

    positions = survey.electrode_positions[:, :2]
    cell_ids, _ = locate_points(mesh.nodes, mesh.cells, positions)
    distance = np.linalg.norm(mesh.nodes[None] - positions[:, None], axis=2)
    nearest = np.argmin(distance, axis=1)
    nodes = np.where(distance[np.arange(len(positions)), nearest] <= 1e-2, nearest, -1)
    ptr, lists = [0], []
    for e, node in enumerate(nodes):
        around = np.flatnonzero((mesh.cells == node).any(axis=1)) if node >= 0 else np.asarray([cell_ids[e]])
        lists.append(around)
        ptr.append(ptr[-1] + len(around))
    return nodes, cell_ids, np.asarray(ptr, dtype=np.int32), np.ascontiguousarray(np.concatenate(lists), dtype=np.int32)


def space_problem(d: Discretization, mesh: Mesh, survey: Survey, k: np.ndarray, w: np.ndarray) -> ProblemArrays:
    """Plan arrays of any discretization (terrain auxiliary spaces: parent cells, quadratic
    elements, dense electrode rows turned into receiver lists)."""

    rows = d.electrode_matrix
    width = max(int(np.max(np.count_nonzero(rows, axis=1))), 1)
    rdofs = np.full((rows.shape[0], width), -1, dtype=np.int32)
    rw = np.zeros((rows.shape[0], width))
    for e, row in enumerate(rows):
        nz = np.flatnonzero(row)
        rdofs[e, :len(nz)], rw[e, :len(nz)] = nz, row[nz]
    src_nodes, src_cells, sptr, scells = source_cells(mesh, survey)
    K, BL = d.cell_dofs.shape[1], d.boundary_dofs.shape[1]
    arrays = {
        "coords": np.ascontiguousarray(d.dof_nodes, dtype=np.float64),
        "cell_dofs": np.ascontiguousarray(d.cell_dofs, dtype=np.int32),
        "stiffness": np.ascontiguousarray(d.stiffness, dtype=np.float64),
        "mass": np.ascontiguousarray(d.mass, dtype=np.float64),
        "parents": np.ascontiguousarray(d.parent_cell_ids, dtype=np.int32),
        "bdofs": np.ascontiguousarray(d.boundary_dofs, dtype=np.int32),
        "bcells": np.ascontiguousarray(d.boundary_cells, dtype=np.int32),
        "bmass": np.ascontiguousarray(d.boundary_mass, dtype=np.float64),
        "bcoef": np.ascontiguousarray(d.boundary_geometries, dtype=np.float64),
        "k": np.ascontiguousarray(k, dtype=np.float64),
        "w": np.ascontiguousarray(w, dtype=np.float64),
        "rdofs": rdofs,
        "rw": rw,
        "abmn": np.ascontiguousarray(survey.measurement_slots(), dtype=np.int32),
        "sptr": sptr,
        "scells": scells,
    }
    counts = {"N": d.dof_count, "C": len(d.cell_dofs), "Cm": mesh.cell_count, "K": K, "BL": BL, "RW": width,
              "Nb": len(d.boundary_dofs), "W": len(k), "E": survey.electrode_count, "D": survey.measurement_count}
    return ProblemArrays(arrays, k, w, d.stiffness, d.mass, d.boundary_mass, d.boundary_geometries,
                         d.electrode_matrix, src_nodes, src_cells, counts)


TERRAIN_CACHE_VERSION = "b200_terrain_unit_potentials_v1"


def _terrain_cache_dir(value) -> Path | None:
    """Folder of the terrain unit-potential cache: the argument, else ``ADTLERT_TERRAIN_CACHE_DIR``
    (unset or empty: no disk cache) (adtlert/forward/ert2p5d.py:1135-1145)."""

    if value is not None:
        return Path(value).expanduser()
    env = os.environ.get("ADTLERT_TERRAIN_CACHE_DIR", "").strip()
    return Path(env).expanduser() if env else None


JACOBIAN_CHUNKS = 8
"""Column chunks of a Jacobian computed straight into host memory (copy of chunk k overlaps
the computation of chunk k + 1)."""


def _to_host(tensor: Tensor) -> Tensor:
    """Device tensor -> CPU tensor in page-locked memory (torch's caching host allocator), so the
    copy runs at full link bandwidth."""

    out = torch.empty(tensor.shape, dtype=tensor.dtype, pin_memory=True)
    out.copy_(tensor, non_blocking=True)
    torch.cuda.current_stream(tensor.device).synchronize()
    return out


def _widened_to_host(tensor: Tensor, dtype: torch.dtype = torch.float64, chunk_bytes: int = 256 << 20) -> Tensor:
    """Device matrix -> page-locked CPU matrix of a wider dtype, widened on the device a block of
    rows at a time, so the device holds at most ``chunk_bytes`` of the wide copy beside the
    original (a whole-matrix widening would need three times the float32 matrix)."""

    rows, columns = int(tensor.shape[0]), int(tensor.shape[1])
    out = torch.empty(tensor.shape, dtype=dtype, pin_memory=True)
    step = max(1, chunk_bytes // max(1, columns * (torch.finfo(dtype).bits // 8)))
    buffers = []
    for r0 in range(0, rows, step):
        wide = tensor[r0:r0 + step].to(dtype)
        out[r0:r0 + step].copy_(wide, non_blocking=True)
        buffers.append(wide)  # kept alive until the copies finish
        if len(buffers) > 2:  # at most two chunks in flight
            torch.cuda.current_stream(tensor.device).synchronize()
            buffers = buffers[-1:]
    torch.cuda.current_stream(tensor.device).synchronize()
    return out


def _checked_to_host(tensor: Tensor, context: str) -> Tensor:
    """``_to_host`` with the finiteness check done on the device, queued before the copy, so a
    large result is never scanned on the host."""

    finite = finite_flag(tensor)
    out = _to_host(tensor)
    if not bool(finite):
        raise FloatingPointError(f"{context} produced non-finite values")
    return out


def _mesh_arrays(mesh) -> Mesh:
    """Our Mesh for the reference's or our own mesh object."""

    if isinstance(mesh, Mesh):
        return mesh
    surface = getattr(mesh, "surface_node_ids", None)
    return Mesh.from_arrays(mesh.nodes, mesh.cells, surface_node_ids=surface)


def _survey_arrays(survey) -> Survey:
    if isinstance(survey, Survey):
        return survey
    return Survey.from_arrays(survey.electrode_positions, survey.measurements)


class ERTForward2p5D:
    """2.5D ERT forward operator (analytic primary field on flat surfaces, numerical primary
    field on terrain) on B200 kernels."""

    def __init__(
        self,
        mesh,
        survey,
        *,
        quadrature_order: int = 2,
        numerical_h2_refined: bool = True,
        numerical_p2_refined: bool = True,
        topographic_geometric_factor_mode: str = "analytic",
        terrain_cache_dir=None,
        normal_field_cache_max_entries: int = 8,
        series_batch_steps: int = 8,
    ) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("ADTLERT requires an NVIDIA GPU with CUDA (B200 kernels)")
        gf_mode = option(topographic_geometric_factor_mode, ("analytic", "numerical"), "topographic_geometric_factor_mode")
        if int(normal_field_cache_max_entries) < 0:
            raise ValueError("normal_field_cache_max_entries must be non-negative")
        if int(series_batch_steps) < 1:
            raise ValueError("series_batch_steps must be >= 1")
        self.source_mesh, self.source_survey = mesh, survey
        self.mesh = _mesh_arrays(mesh)
        self.survey = _survey_arrays(survey)
        self.numerical_h2_refined = bool(numerical_h2_refined)
        self.numerical_p2_refined = bool(numerical_p2_refined)
        self.topographic_geometric_factor_mode = gf_mode
        self.terrain_cache_dir = _terrain_cache_dir(terrain_cache_dir)
        self._terrain = not self.mesh.is_flat_surface
        self.normal_field_cache_max_entries = int(normal_field_cache_max_entries)
        self.series_batch_steps = int(series_batch_steps)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = _native.load_library()
        self._cache: dict = {}
        self._field_cache = FieldStore(self.normal_field_cache_max_entries, self._fingerprints)
        self._pending_checks = None  # (device flag, context) pairs read back with a host result
        self._solver = _Slots()
        self._plan = None
        self._build(int(quadrature_order))

    @classmethod
    def from_mesh_survey(cls, mesh, survey, quadrature_order: int = 2, numerical_h2_refined: bool = True,
                         numerical_p2_refined: bool = True, topographic_geometric_factor_mode: str = "analytic",
                         terrain_cache_dir=None, normal_field_cache_max_entries: int = 8,
                         series_batch_steps: int = 8) -> ERTForward2p5D:
        return cls(
            mesh,
            survey,
            quadrature_order=quadrature_order,
            numerical_h2_refined=numerical_h2_refined,
            numerical_p2_refined=numerical_p2_refined,
            topographic_geometric_factor_mode=topographic_geometric_factor_mode,
            terrain_cache_dir=terrain_cache_dir,
            normal_field_cache_max_entries=normal_field_cache_max_entries,
            series_batch_steps=series_batch_steps,
        )

    # ------------------------------------------------------------------ set-up
    def _build(self, quadrature_order: int) -> None:
        mesh, survey = self.mesh, self.survey
        E, D = survey.electrode_count, survey.measurement_count
        if self._terrain:
            k, w = inverse_cosine_weights(*wavenumber_bounds(survey.electrode_positions))
            refine = self.numerical_h2_refined

            def build(name, **options):
                return build_discretization(name, mesh, survey, k, auxiliary=True, refine=refine,
                                            quadrature_order=quadrature_order, **options)

            self.discretization = build("primary")
            self.primary_potential_discretization = build("primary_potential", quadratic=True)
            self.geometric_discretization = None
            if self.topographic_geometric_factor_mode == "numerical":
                self.geometric_discretization = build("geometric", quadratic=self.numerical_p2_refined)
            problem = space_problem(self.discretization, mesh, survey, k, w)
        else:
            problem = build_problem(mesh, survey, quadrature_order)
            k, w = problem.wavenumbers, problem.weights
            self.primary_potential_discretization = self.geometric_discretization = None
        self._problem = problem
        self.wavenumbers = torch.as_tensor(k, dtype=FLOAT_DTYPE)
        self.weights = torch.as_tensor(w, dtype=FLOAT_DTYPE)
        self.source_node_ids = torch.as_tensor(problem.source_nodes, dtype=torch.long)
        self.source_cell_ids = torch.as_tensor(problem.source_cells, dtype=torch.long)
        self.W, self.E, self.D, self.C = len(k), E, D, mesh.cell_count
        plan, info, order = self._create_plan(problem)
        self._plan = plan
        self.plan_info = info
        self._dof_order = order
        self.N = int(problem.counts["N"])
        self.Cd = int(problem.counts["C"])
        pa = problem
        if not self._terrain:
            self.discretization = Discretization(
                name="native", geometry=mesh, parent_cell_ids=np.arange(mesh.cell_count), dof_nodes=mesh.nodes,
                cell_dofs=mesh.cells, boundary_dofs=mesh.boundary_edges, stiffness=pa.stiffness, mass=pa.mass,
                boundary_mass=pa.boundary_mass, boundary_geometries=pa.robin, electrode_matrix=pa.electrode_matrix,
                spd=True,
            )
            primary = analytic_primary(mesh.nodes, mesh.cells, survey.electrode_positions[:, :2], pa.source_nodes, k)
            self._geometric = torch.as_tensor(geometric_factors(survey.electrode_positions, survey.measurements),
                                              dtype=FLOAT_DTYPE)
        else:
            potential = self.primary_potential_discretization
            selection = exact_node_indices(potential.dof_nodes, self.discretization.dof_nodes)
            primary = self._unit_potentials(potential)[..., selection]
            self._geometric = None
        primary = np.ascontiguousarray(primary, dtype=np.float64)
        with torch.cuda.device(self.device):
            _native.check(self._lib.adt_set_primary(plan, _native.host_ptr(primary), self._stream()), plan, "adt_set_primary")

    def _create_plan(self, problem: ProblemArrays):
        struct = problem.struct()
        plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _native.check(self._lib.adt_plan_create(ctypes.byref(struct), ctypes.byref(plan)), None, "adt_plan_create")
        info = _native.PlanInfo()
        self._lib.adt_plan_get_info(plan, ctypes.byref(info))
        order = np.empty(problem.counts["N"], dtype=np.int32)
        self._lib.adt_plan_dof_order(plan, _native.host_ptr(order))
        return plan, {name: getattr(info, name) for name, _ in _native.PlanInfo._fields_}, order

    # ------------------------------------------------------------------ terrain set-up
    def _disk_path(self, name: str, d: Discretization) -> Path | None:
        if self.terrain_cache_dir is None:
            return None
        digest = hashlib.sha256()
        for label, value in (("version", TERRAIN_CACHE_VERSION), ("name", name),
                             ("options", (self.numerical_h2_refined, self.numerical_p2_refined,
                                          self.topographic_geometric_factor_mode))):
            digest.update(f"{label}={value!r};".encode())
        for array in (self.mesh.nodes, self.mesh.cells, self.mesh.surface_node_ids, self.survey.electrode_positions,
                      self.survey.measurements, self.wavenumbers, self.weights, d.parent_cell_ids, d.dof_nodes,
                      d.cell_dofs, d.boundary_dofs, d.electrode_matrix, d.stiffness, d.mass, d.boundary_mass,
                      d.boundary_geometries):
            array = np.ascontiguousarray(np.asarray(array))
            digest.update(f"{array.dtype}{array.shape}".encode())
            digest.update(array.tobytes())
        return self.terrain_cache_dir / f"{digest.hexdigest()}.npz"

    def _unit_potentials(self, d: Discretization) -> np.ndarray:
        """Unit-conductivity potentials (W, E, dofs) of every electrode on ``d``: A_w(1) u = Pel
        for every wavenumber, float64, a few wavenumbers per factorization; cached per
        discretization in memory and, with a cache folder, on disk (ert2p5d.py:349-416)."""

        key = ("unit_potentials", d.name)
        if key in self._cache:
            return self._cache[key]
        shape = (self.W, self.E, d.dof_count)
        path = self._disk_path(f"{d.name}_unit_potentials", d)
        value = None
        if path is not None and path.exists():
            with contextlib.suppress(Exception):
                with np.load(path) as stored:
                    value = stored["value"] if stored["value"].shape == shape else None
        if value is None:
            value = self._solve_unit_potentials(d)
            if path is not None:
                with contextlib.suppress(OSError):
                    path.parent.mkdir(parents=True, exist_ok=True)
                    tmp = path.with_name(f"{path.name}.{os.getpid()}.tmp.npz")
                    np.savez(tmp, value=value)
                    tmp.replace(path)
        self._cache[key] = value
        return value

    def _solve_unit_potentials(self, d: Discretization) -> np.ndarray:
        problem = space_problem(d, self.mesh, self.survey, self.wavenumbers.double().numpy(),
                                self.weights.double().numpy())
        plan, info, order = self._create_plan(problem)
        lib, N, E, W = self._lib, d.dof_count, self.E, self.W
        try:
            with torch.cuda.device(self.device):
                stream = self._stream()
                ones = torch.ones((1, self.C), dtype=torch.float32, device=self.device)
                free, _ = torch.cuda.mem_get_info(self.device)
                per_system = 8.0 * (info["factor_doubles_per_system"] + info["nnz"] + 2 * N * E)
                chunk = int(max(1, min(W, 0.4 * free // max(per_system, 1.0))))
                rows = torch.as_tensor(np.ascontiguousarray(d.electrode_matrix.T[order]), device=self.device)
                solver_position = torch.as_tensor(np.argsort(order), device=self.device)  # dof -> solver row
                out = torch.empty((W, E, N), dtype=torch.float64)
                finite = torch.ones((), dtype=torch.bool, device=self.device)
                for w0 in range(0, W, chunk):
                    count = min(chunk, W - w0)
                    _native.check(lib.adt_factorize_wavenumbers(plan, 0, _native.ptr(ones), w0, count, stream), plan,
                                  "adt_factorize_wavenumbers")
                    rhs = rows[None].repeat(count, 1, 1).contiguous()
                    _native.check(lib.adt_solve(plan, 0, count, E, _native.ptr(rhs), stream), plan, "adt_solve")
                    # (count, N solver order, E) -> (count, E, N dof order) on the device
                    solved = rhs.index_select(1, solver_position).transpose(1, 2).contiguous()
                    del rhs
                    finite &= finite_flag(solved)
                    out[w0:w0 + count].copy_(solved)
                if not bool(finite):
                    raise FloatingPointError("unit potentials: non-finite values")
                return out.numpy()
        finally:
            torch.cuda.synchronize(self.device)
            lib.adt_plan_destroy(plan)

    def _numerical_geometric_factors(self) -> Tensor:
        """1 / (normal transfer of the unit-conductivity potentials on the geometric
        discretization) (ert2p5d.py:697-706)."""

        d = self.geometric_discretization
        potential = self.primary_potential_discretization
        same = (d.dof_count == potential.dof_count and np.array_equal(d.cell_dofs, potential.cell_dofs)
                and np.array_equal(d.dof_nodes, potential.dof_nodes))
        units = self._unit_potentials(potential if same else d)
        integrated = np.tensordot(self.weights.double().numpy(), units, axes=([0], [0]))  # (E, dofs)
        table = np.zeros((self.E + 1, self.E + 1))
        table[:self.E, :self.E] = integrated @ d.electrode_matrix.T
        a, b, m, n = self.survey.measurement_slots().T
        sources = table[a] - table[b]
        rows = np.arange(self.D)
        return torch.as_tensor(1.0 / (sources[rows, m] - sources[rows, n]), dtype=torch.float64)

    # ------------------------------------------------------------------ helpers
    def _stream(self):
        return _native.stream_handle(self.device)

    @property
    def dtype(self) -> torch.dtype:
        """Result precision: float64 on terrain (as the reference), ``FLOAT_DTYPE`` otherwise."""

        return torch.float64 if self._terrain else FLOAT_DTYPE

    @property
    def use_numerical_primary(self) -> bool:
        return self.primary_potential_discretization is not None

    @property
    def use_numerical_geometric_factors(self) -> bool:
        return self.geometric_discretization is not None

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

    def _sigma(self, conductivity) -> Tensor:
        return conductivity_model(conductivity, self.C)

    def _series(self, conductivities) -> Tensor:
        return conductivity_series(conductivities, self.C)

    def _geometric_factors(self) -> Tensor:
        if self._geometric is None:
            if self.use_numerical_geometric_factors:
                self._geometric = self._numerical_geometric_factors()
            else:
                self._geometric = torch.as_tensor(
                    geometric_factors(self.survey.electrode_positions, self.survey.measurements), dtype=FLOAT_DTYPE)
        return self._geometric

    def _call(self, name: str, *args) -> None:
        _native.check(getattr(self._lib, name)(self._plan, *args), self._plan, name)

    def _factorize(self, sigmas: Tensor, name) -> int:
        """Slot holding the factorization of ``sigmas`` (device float32, (B, C)); refactorizes
        unless the slot of this batch size already holds the named factorization."""

        batch = int(sigmas.shape[0])
        entry = self._solver.lookup(batch)
        if not self._solver.holds(batch, name):
            self._call("adt_factorize", entry["slot"], _native.ptr(sigmas), batch, self._stream())
            entry["name"] = name
            self._solver.factorizations += 1
        return entry["slot"]

    # ------------------------------------------------------------------ fields
    def _solve_fields(self, sigmas: Tensor, name) -> list[_Fields]:
        batch = int(sigmas.shape[0])
        sig = sigmas.to(self.device, torch.float32, non_blocking=True).contiguous()
        entry = self._solver.lookup(batch)
        # the factorization also forward-reduces the field right-hand sides solved just below
        self._call("adt_factorize_fields", entry["slot"], _native.ptr(sig), batch, self._stream())
        entry["name"] = name
        self._solver.factorizations += 1
        total = torch.empty((batch, self.W, self.N, self.E), dtype=torch.float32, device=self.device)
        self._call("adt_solve_fields", entry["slot"], _native.ptr(sig), batch, _native.ptr(total), self._stream())
        if self._pending_checks is not None:
            self._pending_checks.append((torch.isfinite(total).all(), "total fields"))
        else:
            check_finite(total, "total fields")
        return [_Fields(total[i]) for i in range(batch)]

    @contextlib.contextmanager
    def _deferred_checks(self):
        """Finiteness checks of solved fields queued on the device and read after the block, whose
        result copy synchronizes anyway; on a failure the field cache is cleared (so non-finite
        fields are never served later) and the same FloatingPointError is raised."""

        self._pending_checks = []
        try:
            yield
            pending = self._pending_checks
        finally:
            self._pending_checks = None
        if pending and not bool(torch.stack([flag for flag, _ in pending]).all()):
            self._field_cache.clear()
            context = next(what for flag, what in pending if not bool(flag))
            raise FloatingPointError(f"{context} produced non-finite values")

    def _fingerprints(self, models: Tensor) -> list[bytes]:
        return model_fingerprints(self._lib, self._plan, models, self._stream())

    def _fields_series(self, models: Tensor):
        return self._field_cache.fields(models, self.series_batch_steps, self._solve_fields)

    def _fields(self, conductivity) -> _Fields:
        return self._fields_series(self._sigma(conductivity)[None])[0][0]

    def normal_field_cache_info(self) -> dict[str, int]:
        return self._field_cache.info()

    def _stack(self, fields: list[_Fields]) -> Tensor:
        if len(fields) == 1:
            return fields[0].total[None]
        return torch.stack([f.total for f in fields]).contiguous()

    def _transfers(self, totals: Tensor, potentials: bool = False):
        """Normal and reciprocal transfers (S, D) float64 on the device (+ (S, E, E) potentials)."""

        S = int(totals.shape[0])
        normal = torch.empty((S, self.D), dtype=torch.float64, device=self.device)
        reciprocal = torch.empty_like(normal)
        pot = torch.empty((S, self.E, self.E), dtype=torch.float64, device=self.device) if potentials else None
        self._call("adt_measure", _native.ptr(totals), S, _native.ptr(normal), _native.ptr(reciprocal), _native.ptr(pot), self._stream())
        return normal, reciprocal, pot

    @staticmethod
    def _combine(normal: Tensor, reciprocal: Tensor) -> Tensor:
        return torch.sign(normal) * torch.sqrt(torch.abs(normal * reciprocal))

    def _measure(self, conductivity):
        fields = self._fields(conductivity)
        normal, reciprocal, _ = self._transfers(fields.total[None])
        return fields, normal[0], reciprocal[0]

    # ------------------------------------------------------------------ forward API
    def solve(self, conductivity, currents=1.0) -> ForwardResponse:
        fields = self._fields(conductivity)
        normal, reciprocal, potentials = self._transfers(fields.total[None], potentials=True)
        return self._response(fields, normal[0], reciprocal[0], potentials[0], currents)

    def _response(self, fields, normal, reciprocal, potentials, currents) -> ForwardResponse:
        integrated = torch.empty((self.E, self.N), dtype=torch.float32, device=self.device)
        self._call("adt_integrated_potentials", _native.ptr(fields.total), _native.ptr(integrated), self._stream())
        check_finite(integrated, "integrated potentials")
        resistance = self._combine(normal.cpu(), reciprocal.cpu()).to(self.dtype)
        current = torch.as_tensor(currents, dtype=FLOAT_DTYPE)
        if potentials is None:
            _, _, pot = self._transfers(fields.total[None], potentials=True)
            potentials = pot[0]
        return ForwardResponse(
            apparent_resistivity=self._geometric_factors() * resistance / current,
            resistance=resistance,
            electrode_potentials=potentials.cpu().to(self.dtype),
            integrated_potentials=integrated.cpu().to(self.dtype),
            wavenumbers=self.wavenumbers,
            weights=self.weights,
        )

    def resistance(self, conductivity) -> Tensor:
        _, normal, reciprocal = self._measure(conductivity)
        return self._combine(normal.cpu(), reciprocal.cpu()).to(self.dtype)

    def apparent_resistivity_values(self, conductivity, currents=1.0) -> Tensor:
        current = torch.as_tensor(currents, dtype=FLOAT_DTYPE)
        return self._geometric_factors() * self.resistance(conductivity) / current

    def resistance_series(self, conductivities) -> Tensor:
        return self._resistances_device(self._series(conductivities)).cpu()

    def _resistances_device(self, models: Tensor) -> Tensor:
        """Reciprocity-averaged resistances (S, D) of validated models (S, C), left on the GPU in
        the operator's result dtype."""

        fields, _ = self._fields_series(models)
        normal, reciprocal, _ = self._transfers(self._stack(fields))
        return self._combine(normal, reciprocal).to(self.dtype)

    def apparent_resistivity_series(self, conductivities, currents=1.0) -> Tensor:
        current = torch.as_tensor(currents, dtype=FLOAT_DTYPE)
        resistance = self.resistance_series(conductivities)
        if current.ndim == 1 and current.shape[0] == resistance.shape[0] and current.shape[0] != resistance.shape[1]:
            current = current[:, None]
        return self._geometric_factors() * resistance / current

    def prepare(self, conductivity=None, *, include_solver_state: bool = True) -> None:
        """Populate the geometric factors and, optionally, the solver and field caches before
        timed solves (the rest of the set-up is done at construction)."""

        self._geometric_factors()
        if include_solver_state:
            self._fields(torch.ones(self.C) if conductivity is None else conductivity)

    # ------------------------------------------------------------------ derivatives
    def _columns(self, cell_parameter_ids=None, parameter_count=None, discretization: bool = False):
        """(key, columns, ptr, cells) of the aggregation of model cells (or, with
        ``discretization``, of the discretization's cells through their parents) into parameters,
        or None for the identity (ert2p5d.py:751-763)."""

        ids, count = parameter_targets(cell_parameter_ids, parameter_count, self.C)
        refined = discretization and self.Cd != self.C
        if cell_parameter_ids is None and not refined:
            return None
        if refined:
            ids = ids[self.discretization.parent_cell_ids]
        digest = hashlib.blake2b(np.ascontiguousarray(ids).tobytes(), digest_size=16).digest()
        key = ("columns", digest, count, len(ids))
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

    def _batch_size(self, batch_size, direct: bool) -> int:
        if batch_size is None:
            if not direct:
                return 8
            return min(self.D, 64) if self.C >= 4096 else self.D
        if batch_size < 1:
            raise ValueError("batch_size must be >= 1")
        return int(batch_size)

    def _jacobian_device(self, fields: _Fields, columns=None) -> Tensor:
        """Normal-quadrupole Jacobian (D, C or P) on the device; every row in one launch over the
        discretization's cells, then summed into model cells or parameters."""

        J = torch.empty((self.D, self.Cd), dtype=torch.float32, device=self.device)
        self._call("adt_normal_jacobian", _native.ptr(fields.total), 0, self.D, _native.ptr(J), self._stream())
        return self._aggregate(J, columns)

    def solve_with_jacobian(self, conductivity, currents=1.0, *, batch_size=None,
                            include_robin_boundary_derivative: bool = False, normal_sensitivity: bool = True,
                            jacobian_cell_parameter_ids=None, jacobian_parameter_count=None):
        response, jacobian = self._solve_with_jacobian_device(
            conductivity, currents, batch_size=batch_size,
            include_robin_boundary_derivative=include_robin_boundary_derivative,
            normal_sensitivity=normal_sensitivity, jacobian_cell_parameter_ids=jacobian_cell_parameter_ids,
            jacobian_parameter_count=jacobian_parameter_count)
        return response, _widened_to_host(jacobian, self.dtype)  # widened on the device: exact, and cheaper

    def _solve_with_jacobian_device(self, conductivity, currents=1.0, *, batch_size=None,
                                    include_robin_boundary_derivative: bool = False, normal_sensitivity: bool = True,
                                    jacobian_cell_parameter_ids=None, jacobian_parameter_count=None):
        """The response (CPU) and the Jacobian still on the device (float32)."""

        fields, normal, reciprocal = self._measure(conductivity)
        direct = normal_sensitivity and not include_robin_boundary_derivative
        batch = self._batch_size(batch_size, direct)
        if direct:
            columns = self._columns(jacobian_cell_parameter_ids, jacobian_parameter_count, discretization=True)
            jacobian = self._jacobian_device(fields, columns)
        else:
            key = self._field_cache.key(self._sigma(conductivity))
            slot = self._factorize(self._sigma(conductivity).to(self.device)[None].contiguous(), batch_name([key]))
            rows = []
            for start in range(0, self.D, batch):
                count = min(batch, self.D - start)
                out = torch.empty((count, self.C), dtype=torch.float32, device=self.device)
                self._call("adt_adjoint_jacobian", slot, _native.ptr(fields.total), _native.ptr(normal), _native.ptr(reciprocal),
                           start, count, int(include_robin_boundary_derivative), int(normal_sensitivity), _native.ptr(out), self._stream())
                rows.append(out)
            jacobian = torch.cat(rows) if len(rows) > 1 else rows[0]
        return self._response(fields, normal, reciprocal, None, currents), jacobian

    def jacobian(self, conductivity, *, batch_size=None, include_robin_boundary_derivative: bool = False,
                 normal_sensitivity: bool = True) -> Tensor:
        """The Jacobian of ``solve_with_jacobian`` without the response: on the direct path only the
        fields and J are computed, and J's copy to the host is the call's one synchronization."""

        direct = normal_sensitivity and not include_robin_boundary_derivative
        if not direct:
            return self.solve_with_jacobian(conductivity, batch_size=batch_size,
                                            include_robin_boundary_derivative=include_robin_boundary_derivative,
                                            normal_sensitivity=normal_sensitivity)[1]
        self._batch_size(batch_size, direct)
        with self._deferred_checks():
            fields = self._fields(conductivity)
            columns = self._columns(None, None, discretization=True)
            if columns is None:
                host = self._jacobian_to_host(fields)
            else:  # float64 results (terrain) are widened on the device, not over the host's memory
                host = _widened_to_host(self._jacobian_device(fields, columns), self.dtype)
        return host.to(self.dtype)

    def _jacobian_to_host(self, fields: _Fields) -> Tensor:
        """J (D, C) in page-locked host memory: computed in column chunks whose copies to the host
        overlap the computation of the next chunk (adt_normal_jacobian_to_host)."""

        J = torch.empty((self.D, self.Cd), dtype=torch.float32, device=self.device)
        host = torch.empty((self.D, self.Cd), dtype=torch.float32, pin_memory=True)
        self._call("adt_normal_jacobian_to_host", _native.ptr(fields.total), _native.ptr(J), _native.ptr(host),
                   JACOBIAN_CHUNKS, self._stream())
        torch.cuda.current_stream(self.device).synchronize()
        return host

    def jacobian_columnwise(self, conductivity) -> Tensor:
        basis = torch.eye(self.C, dtype=self.dtype)
        return torch.stack([self.jvp(conductivity, column) for column in basis], dim=1)

    def vjp(self, conductivity, cotangent) -> Tensor:
        cotangent = measurement_vector(cotangent, self.D, FLOAT_DTYPE)
        return self.vjp_series(self._sigma(conductivity)[None], cotangent[None])[0]

    def vjp_series(self, conductivities, cotangents) -> Tensor:
        models = self._series(conductivities)
        cotangents = cotangent_series(cotangents, models.shape[0], self.D)
        gradient = self._vjp_device(models, cotangents).cpu().to(self.dtype)
        check_finite(gradient, "conductivity gradient")
        return gradient

    def _vjp_device(self, models: Tensor, cotangents: Tensor) -> Tensor:
        """Exact VJPs (S, C) float32 on the GPU of validated models (S, C) and resistance
        cotangents (S, D) on any device."""

        fields, keys = self._fields_series(models)
        gradients: dict[int, Tensor] = {}
        for batch in adjoint_batches(len(fields), self.series_batch_steps):
            totals = self._stack([fields[step] for step in batch])
            normal, reciprocal, _ = self._transfers(totals)
            slot = self._factorize(models[batch].to(self.device, torch.float32).contiguous(),
                                   batch_name([keys[step] for step in batch]))
            cot = cotangents[batch].to(self.device, torch.float64).contiguous()
            grad = torch.empty((len(batch), self.C), dtype=torch.float32, device=self.device)
            self._call("adt_vjp", slot, _native.ptr(totals), _native.ptr(normal), _native.ptr(reciprocal),
                       _native.ptr(cot), len(batch), _native.ptr(grad), self._stream())
            for i, step in enumerate(batch):
                gradients[step] = grad[i]
        return torch.stack([gradients[step] for step in range(len(fields))])

    def jvp(self, conductivity, delta_conductivity) -> Tensor:
        out = self._jvp_device(self._sigma(conductivity), cell_vector(delta_conductivity, self.C))
        check_finite(out, "tangent fields")
        return out.cpu().to(self.dtype)

    def _jvp_device(self, sigma: Tensor, direction: Tensor) -> Tensor:
        """Resistance tangent (D,) float64 on the GPU of a validated model and direction (C,)."""

        fields, normal, reciprocal = self._measure(sigma)
        direction = direction.to(self.device, torch.float32).contiguous()
        slot = self._factorize(sigma.to(self.device)[None].contiguous(), batch_name([self._field_cache.key(sigma)]))
        out = torch.empty(self.D, dtype=torch.float64, device=self.device)
        self._call("adt_jvp", slot, _native.ptr(fields.total), _native.ptr(normal), _native.ptr(reciprocal),
                   _native.ptr(direction), _native.ptr(out), self._stream())
        return out

    def normal_vjp(self, conductivity, cotangent, *, cell_parameter_ids=None, parameter_count=None) -> Tensor:
        columns = self._columns(cell_parameter_ids, parameter_count)
        fields = self._fields(conductivity)
        weights = measurement_vector(cotangent, self.D, torch.float64).to(self.device).contiguous()
        grad = torch.empty((1, self.C), dtype=torch.float32, device=self.device)
        self._call("adt_normal_vjp", _native.ptr(fields.total), _native.ptr(weights), 0, _native.ptr(grad), self._stream())
        gradient = self._aggregate(grad, columns)[0].cpu().to(self.dtype)
        check_finite(gradient, "normal sensitivity vjp")
        return gradient

    def normal_vjp_series(self, conductivities, cotangents, *, cell_parameter_ids=None, parameter_count=None) -> Tensor:
        models = self._series(conductivities)
        cotangents = cotangent_series(cotangents, models.shape[0], self.D)
        return torch.stack([
            self.normal_vjp(m, c, cell_parameter_ids=cell_parameter_ids, parameter_count=parameter_count)
            for m, c in zip(models, cotangents, strict=True)
        ])

    def normal_jvp(self, conductivity, delta_conductivity) -> Tensor:
        fields = self._fields(conductivity)
        direction = cell_vector(delta_conductivity, self.C).to(self.device, torch.float32).contiguous()
        out = torch.empty(self.D, dtype=torch.float64, device=self.device)
        self._call("adt_normal_jvp", _native.ptr(fields.total), _native.ptr(direction), 0, _native.ptr(out), self._stream())
        result = out.cpu().to(self.dtype)
        check_finite(result, "normal sensitivity jvp")
        return result

    # ------------------------------------------------------------------ lifetime
    def close(self) -> None:
        """Drop cached fields and forget held factorizations (the operator keeps working)."""

        self._field_cache.clear()
        self._solver.close()

    def __del__(self) -> None:
        with contextlib.suppress(Exception):
            if self._plan is not None:
                torch.cuda.synchronize(self.device)
                self._lib.adt_plan_destroy(self._plan)
                self._plan = None
