"""The reference's own GPU kernel, built for timing and parity (TEST INFRASTRUCTURE ONLY).

AD-TLERT ships one CUDA kernel, ``normal_sensitivity<T, K>`` (adtlert/forward/kernels.py:132-178).
The reference compiles it at run time with NVRTC for the current device (kernels.py:196-219:
``arch=sm_<major><minor>``, C++17, ``BLOCK_CELLS=32``, ``BLOCK_DATA=4``) and launches one thread
per (row, cell) entry on blocks of 32 cells x 4 rows (kernels.py:222-268), 64 rows per launch
for sections of 4096 cells or more (ert2p5d.py:971-1010).

``build(reference_root)`` reads that source string out of the reference's file where it lies
(it is never copied into this repository), writes it beside a launcher of our own into
``oracle/_ref/`` (git-ignored) and compiles both with nvcc for ``sm_100``, the target NVRTC
picks on a B200. The resulting ``oracle/_ref/libnormal_sensitivity_ref.so`` travels with the
tree, so the benchmark and the GPU test need only that file. ``load()`` opens it.

Run as ``python oracle/reference_kernel.py <reference root>`` (``__graft_entry__.build()`` does
this when the reference tree is present).
"""

from __future__ import annotations

import ast
import ctypes
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIBRARY = OUT / "libnormal_sensitivity_ref.so"
KERNEL_FILE = Path("adtlert") / "forward" / "kernels.py"

# Launcher of our own around the reference's template. The (dtype, K) pairs cover the P1/P2
# triangles, Q1/serendipity quads and P1/P2 tetrahedra the operators use.
_LAUNCHER = r"""
#include <cuda_runtime.h>
#include "reference_source.cuh"

template <typename T, int K>
static int run(const void* phi, const void* a, const void* b, const void* m, const void* n,
               const void* cells, const void* templates, void* out, int W, int S, long long N,
               int D, int C, void* stream)
{
    if (C <= 0 || D <= 0) return 0;
    const long long blocks = (long long)((C + BLOCK_CELLS - 1) / BLOCK_CELLS) *
                             ((D + BLOCK_DATA - 1) / BLOCK_DATA);
    if (blocks > 2147483647LL) return (int)cudaErrorInvalidConfiguration;
    normal_sensitivity<T, K><<<(unsigned)blocks, dim3(BLOCK_CELLS, BLOCK_DATA), 0,
                               (cudaStream_t)stream>>>(
        (const T*)phi, (const int*)a, (const int*)b, (const int*)m, (const int*)n,
        (const int*)cells, (const T*)templates, (T*)out, W, S, N, D, C);
    return (int)cudaGetLastError();
}

extern "C" int adtref_normal_sensitivity(int element_bytes, int K, const void* phi, const void* a,
                                         const void* b, const void* m, const void* n,
                                         const void* cells, const void* templates, void* out,
                                         int W, int S, long long N, int D, int C, void* stream)
{
#define ADTREF_CASE(T, KK) \
    if (element_bytes == (int)sizeof(T) && K == KK) \
        return run<T, KK>(phi, a, b, m, n, cells, templates, out, W, S, N, D, C, stream);
    ADTREF_CASE(float, 3) ADTREF_CASE(float, 4) ADTREF_CASE(float, 6) ADTREF_CASE(float, 8)
    ADTREF_CASE(float, 10) ADTREF_CASE(double, 3) ADTREF_CASE(double, 4) ADTREF_CASE(double, 6)
    ADTREF_CASE(double, 8) ADTREF_CASE(double, 10)
#undef ADTREF_CASE
    return (int)cudaErrorInvalidValue;
}
"""


def _assignments(path: Path) -> dict:
    """Module-level literal assignments of ``path`` (read as text, never imported)."""

    found = {}
    for node in ast.parse(path.read_text()).body:
        if not isinstance(node, ast.Assign):
            continue
        for target in node.targets:
            if isinstance(target, ast.Name):
                try:
                    found[target.id] = ast.literal_eval(node.value)
                except ValueError:
                    pass
            elif isinstance(target, ast.Tuple) and isinstance(node.value, ast.Tuple):
                for name, value in zip(target.elts, node.value.elts):
                    if isinstance(name, ast.Name):
                        try:
                            found[name.id] = ast.literal_eval(value)
                        except ValueError:
                            pass
    return found


def build(reference_root: str | Path, nvcc: str = "nvcc") -> Path:
    """Compile the reference kernel from ``<reference_root>/adtlert/forward/kernels.py``."""

    source_file = Path(reference_root) / KERNEL_FILE
    values = _assignments(source_file)
    source = values["_SENSITIVITY_SOURCE"]
    block_cells, block_data = int(values["_BLOCK_CELLS"]), int(values["_BLOCK_DATA"])
    OUT.mkdir(parents=True, exist_ok=True)
    (OUT / "reference_source.cuh").write_text(source)
    (OUT / "normal_sensitivity_ref.cu").write_text(_LAUNCHER)
    stamp = OUT / "build_flags.txt"
    flags = [nvcc, "-gencode", "arch=compute_100,code=sm_100", "-O3", "-std=c++17",
             f"-DBLOCK_CELLS={block_cells}", f"-DBLOCK_DATA={block_data}", "-Xcompiler", "-fPIC", "-shared",
             "-I", str(OUT), "-o", str(LIBRARY), str(OUT / "normal_sensitivity_ref.cu")]
    subprocess.run(flags, check=True)
    stamp.write_text(" ".join(flags[1:]) + f"\nsource: {KERNEL_FILE}\n")
    return LIBRARY


_lib = None


def available() -> bool:
    return LIBRARY.exists()


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise FileNotFoundError(f"{LIBRARY} is not built (python oracle/reference_kernel.py <reference root>)")
        lib = ctypes.CDLL(str(LIBRARY))
        p = ctypes.c_void_p
        i = ctypes.c_int
        lib.adtref_normal_sensitivity.argtypes = [i, i, p, p, p, p, p, p, p, p, i, i, ctypes.c_longlong, i, i, p]
        lib.adtref_normal_sensitivity.restype = i
        _lib = lib
    return _lib


def normal_sensitivity(phi, a, b, m, n, cells, templates, out, stream=None) -> None:
    """Launch the reference kernel on torch CUDA tensors: ``phi`` (W, S, N), ``templates``
    (W, C, K, K) of the same dtype, ``cells`` (C, K) int32, ABMN int32 (S = remote), ``out``
    (D, C). Queued on ``stream`` (default: torch's current stream)."""

    import torch

    W, S, N = phi.shape
    C, K = cells.shape
    D = a.shape[0]
    for t in (phi, a, b, m, n, cells, templates, out):
        assert t.is_cuda and t.is_contiguous()
    assert templates.shape == (W, C, K, K) and templates.dtype == phi.dtype and out.shape == (D, C)
    handle = (stream or torch.cuda.current_stream(phi.device)).cuda_stream
    ptr = ctypes.c_void_p
    status = load().adtref_normal_sensitivity(
        phi.element_size(), K, *(ptr(t.data_ptr()) for t in (phi, a, b, m, n, cells, templates, out)),
        W, S, N, D, C, ptr(handle))
    if status != 0:
        raise RuntimeError(f"reference normal_sensitivity launch failed (cudaError {status})")


def operator_inputs(forward, fields):
    """The reference kernel's inputs for a flat 2.5D operator of this library and one model's
    total fields ``fields`` ((1, W, N, E) or (W, N, E) float32, solver dof order): ``phi``
    (W, E, N) in the original dof order, templates ``w_w (K_c + k_w^2 M_c)`` (W, C, 3, 3)
    float32 as the reference forms them (ert2p5d.py:984-994), cell dofs and the ABMN slots."""

    import numpy as np
    import torch

    device = fields.device
    total = fields.reshape(-1, *fields.shape[-2:]) if fields.ndim == 4 else fields
    W, N, E = total.shape
    problem = forward._problem
    order = torch.as_tensor(forward._dof_order.astype(np.int64), device=device)
    phi = torch.empty((W, E, N), dtype=torch.float32, device=device)
    phi[:, :, order] = total.permute(0, 2, 1)
    k, w = problem.wavenumbers, problem.weights
    templates = w[:, None, None, None] * (problem.stiffness[None] + (k**2)[:, None, None, None] * problem.mass[None])
    templates = torch.as_tensor(templates, dtype=torch.float32, device=device).contiguous()
    cells = torch.as_tensor(problem.arrays["cell_dofs"], device=device).contiguous()
    abmn = torch.as_tensor(problem.arrays["abmn"], device=device)
    a, b, m, n = (abmn[:, i].contiguous() for i in range(4))
    return phi, a, b, m, n, cells, templates


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python oracle/reference_kernel.py <reference root>")
    print(build(sys.argv[1]))
