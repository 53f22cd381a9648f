"""CPU baselines of the 2.5D Jacobian, flat and terrain (TEST INFRASTRUCTURE ONLY).

The reference's CPU-runnable path for ``jacobian()`` is its assembly, a sparse direct solve per
wavenumber and the normal-sensitivity contraction. Here: the FP64 oracle (``ert2p5d.py``,
SciPy SuperLU per wavenumber) for the flat fields, ``TerrainBaseline`` for terrain sections
(pinned to the reference's terrain Jacobians by the tests), and the C restatement of the
reference kernel (``sensitivity.c``, all host threads) for the contraction.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from .ert2p5d import Oracle2p5D

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_build" / "libsensitivity_cpu.so"


def build() -> Path:
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < (HERE / "sensitivity.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIBRARY


_lib = None


def _library():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build()))
        p = ctypes.c_void_p
        _lib.normal_sensitivity_cpu.argtypes = [p, p, p, p, p, p, p, p, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.normal_sensitivity_cpu.restype = None
    return _lib


def host_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def normal_sensitivity(phi, a, b, m, n, cells, templates, threads: int | None = None) -> np.ndarray:
    """``phi`` (W, S, N) float64; ``templates`` (W, C, K, K); ABMN int arrays (S = remote)."""

    phi = np.ascontiguousarray(phi, dtype=np.float64)
    templates = np.ascontiguousarray(templates, dtype=np.float64)
    cells = np.ascontiguousarray(cells, dtype=np.int32)
    a, b, m, n = (np.ascontiguousarray(v, dtype=np.int32) for v in (a, b, m, n))
    W, S, N = phi.shape
    C, K = cells.shape
    out = np.empty((len(a), C))
    ptr = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _library().normal_sensitivity_cpu(ptr(phi), ptr(a), ptr(b), ptr(m), ptr(n), ptr(cells), ptr(templates), ptr(out),
                                      W, S, N, len(a), C, K, threads or host_threads())
    return out


def jacobian(oracle: Oracle2p5D, sigma, threads: int | None = None) -> np.ndarray:
    """Fields by the oracle (SuperLU), then the C contraction with templates weight_w (K + k_w^2 M)."""

    oracle._fields_cache = {}
    _, total, _ = oracle.fields(np.asarray(sigma, dtype=float))
    templates = oracle.weights[:, None, None, None] * (
        oracle.stiffness[None] + (oracle.wavenumbers**2)[:, None, None, None] * oracle.mass[None]
    )
    a, b, m, n = oracle.slots.T
    return normal_sensitivity(total, a, b, m, n, oracle.cells, templates, threads)


class _Assembly:
    """Matrices A_w(sigma) of a discretization's ``ProblemArrays`` (SciPy CSC, float64): every
    discretization cell carries its parent cell's conductivity, volume terms sigma (K + k^2 M)
    plus the Robin edges sigma alpha_w M_b (adtlert/forward/ert2p5d.py:252-314)."""

    def __init__(self, problem):
        import scipy.sparse as sp

        a, c = problem.arrays, problem.counts
        self.N, self.E, self.W, self.Cm = c["N"], c["E"], c["W"], c["Cm"]
        self.cells = np.ascontiguousarray(a["cell_dofs"], dtype=np.int32)
        self.parents = np.asarray(a["parents"], dtype=np.int64)
        self.k, self.w = np.asarray(a["k"]), np.asarray(a["w"])
        self.stiffness, self.mass = np.asarray(problem.stiffness), np.asarray(problem.mass)
        bdofs = np.asarray(a["bdofs"], dtype=np.int64)
        self.bcell_parents = self.parents[np.asarray(a["bcells"], dtype=np.int64)]
        self.bmass = np.asarray(problem.boundary_mass).reshape(len(bdofs), -1)
        self.bcoef = np.asarray(problem.robin)
        K, BL = self.cells.shape[1], bdofs.shape[1]
        self.rows = np.concatenate((np.repeat(self.cells, K, axis=1).ravel(), np.repeat(bdofs, BL, axis=1).ravel()))
        self.cols = np.concatenate((np.tile(self.cells, (1, K)).ravel(), np.tile(bdofs, (1, BL)).ravel()))
        self._sp = sp

    def matrix(self, sigma, w):
        volume = sigma[self.parents][:, None, None] * (self.stiffness + self.k[w] ** 2 * self.mass)
        boundary = (sigma[self.bcell_parents] * self.bcoef[w])[:, None] * self.bmass
        values = np.concatenate((volume.ravel(), boundary.ravel()))
        return self._sp.csc_matrix((values, (self.rows, self.cols)), shape=(self.N, self.N))


def unit_potentials(problem) -> np.ndarray:
    """Unit-conductivity potentials (W, E, dofs) of every electrode on a discretization's
    ``ProblemArrays``: A_w(1) u = P_el^T per wavenumber, SciPy SuperLU in float64
    (adtlert/forward/ert2p5d.py:349-416, the terrain set-up)."""

    import scipy.sparse.linalg as spl

    assembly = _Assembly(problem)
    rhs = np.asarray(problem.electrode_matrix, dtype=np.float64).T
    ones = np.ones(assembly.Cm)
    return np.stack([spl.splu(assembly.matrix(ones, w)).solve(rhs).T for w in range(assembly.W)])


class TerrainBaseline(_Assembly):
    """FP64 CPU restatement of a terrain operator's ``jacobian()`` (TEST INFRASTRUCTURE ONLY).

    Follows the reference's terrain path (adtlert/forward/ert2p5d.py:328-347, 470-553, 984-1010)
    on the H2-refined field discretization that the library builds bit-identically to the
    reference's (``ProblemArrays`` of ``space_problem``): the secondary right-hand side is
    A(1) u_p - rho_s A(sigma) u_p from the unit potentials u_p of the auxiliary quadratic
    discretization (a set-up product, as the reference caches it), SciPy SuperLU solves every
    wavenumber, and the C contraction (``sensitivity.c``) forms the refined-cell rows, summed
    into model cells.
    """

    def __init__(self, problem, primary):
        super().__init__(problem)
        a = problem.arrays
        self.slots = np.asarray(a["abmn"], dtype=np.int32)
        self.sptr, self.scells = np.asarray(a["sptr"]), np.asarray(a["scells"], dtype=np.int64)
        self.primary = np.asarray(primary, dtype=np.float64)  # (W, E, N)
        # set-up: A_w(1) u_p per wavenumber (the reference's cached reference right-hand side)
        ones = np.ones(self.Cm)
        self.reference_rhs = [self.matrix(ones, w) @ self.primary[w].T for w in range(self.W)]

    def source_resistivities(self, sigma):
        logs = -np.log(sigma[self.scells])
        return np.asarray([np.exp(logs[self.sptr[e]:self.sptr[e + 1]].mean()) for e in range(self.E)])

    def fields(self, sigma):
        """Total potentials (W, E, N) of every electrode source."""

        import scipy.sparse.linalg as spl

        sigma = np.asarray(sigma, dtype=np.float64)
        rho = self.source_resistivities(sigma)
        out = np.empty((self.W, self.E, self.N))
        for w in range(self.W):
            A = self.matrix(sigma, w)
            primary = self.primary[w].T * rho[None, :]
            rhs = self.reference_rhs[w] - A @ primary
            out[w] = (spl.splu(A).solve(rhs) + primary).T
        return out

    def jacobian_rows(self, fields, rows, threads: int | None = None):
        """Rows ``rows`` of the model-cell Jacobian from the fields (refined cells summed)."""

        templates = self.w[:, None, None, None] * (self.stiffness[None] + (self.k**2)[:, None, None, None] * self.mass[None])
        a, b, m, n = self.slots[rows].T
        refined = normal_sensitivity(fields, a, b, m, n, self.cells, templates, threads)
        out = np.zeros((len(rows), self.Cm))
        for d in range(len(rows)):
            out[d] = np.bincount(self.parents, weights=refined[d], minlength=self.Cm)
        return out
