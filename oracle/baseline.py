"""CPU baseline of the flat 2.5D Jacobian (TEST INFRASTRUCTURE ONLY).

The reference's CPU-runnable path for ``jacobian()`` is its assembly, a sparse direct solve per
wavenumber and the normal-sensitivity contraction. Here: the FP64 oracle (``ert2p5d.py``,
SciPy SuperLU per wavenumber) for the fields, and the C restatement of the reference kernel
(``sensitivity.c``, all host threads) for the contraction.
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
