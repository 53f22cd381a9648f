"""ctypes binding of ``libadtlert_b200.so`` (the C ABI declared in ``include/adtlert_b200.h``).

The library is built in-tree (``__graft_entry__.build()`` or ``make -C ad-tlert_b200/csrc``).
There is no fallback: if the library or a CUDA device is missing, the operators raise.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import torch

LIBRARY = Path(__file__).resolve().parent / "libadtlert_b200.so"

ADT_OK, ADT_INVALID_ARG, ADT_NONFINITE, ADT_SOLVER_FAIL, ADT_OOM, ADT_TIMEOUT, ADT_CUDA_ERROR = range(7)

SYMBOLS = (
    "adt_plan_create",
    "adt_plan_destroy",
    "adt_plan_get_info",
    "adt_plan_dof_order",
    "adt_last_error",
    "adt_set_primary",
    "adt_set_static_rhs",
    "adt_factorize",
    "adt_factorize_fields",
    "adt_solve_fields",
    "adt_solve",
    "adt_factorize_wavenumbers",
    "adt_forward",
    "adt_jacobian",
    "adt_measure",
    "adt_integrated_potentials",
    "adt_normal_jacobian",
    "adt_normal_jacobian_to_host",
    "adt_set_jacobian_wait_limit",
    "adt_aggregate_columns",
    "adt_vjp",
    "adt_adjoint_jacobian",
    "adt_jvp",
    "adt_normal_vjp",
    "adt_normal_jvp",
    "adt_boundary_jacobian",
    "adt_measure_static",
    "adt_scale_rows_columns",
    "adt_fingerprint",
    "adt_fingerprint_host",
    "adt_gn_workspace_bytes",
    "adt_gn_step",
    "adt_gn_regularize",
    "adt_mlp_gemm_splits",
    "adt_mlp_gemm",
    "adt_mlp_epilogue",
    "adt_mlp_loss",
    "adt_mlp_bias_grad",
    "adt_mlp_adam",
    "adt_mlp_transpose",
    "adt_mlp_to_bf16",
    "adt_kernel_launches",
    "adt_autotune",
    "adt_get_tuning",
    "adt_set_tuning",
    "adt_jacobian_graph_create",
    "adt_graph_launch",
    "adt_graph_kernels",
    "adt_graph_destroy",
)

JACOBIAN_KERNELS = ("direct", "tc_pipelined", "tc", "fma")

_p = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


class Problem(ctypes.Structure):
    """``adt_problem``: the discretization handed to ``adt_plan_create``."""

    _fields_ = [
        ("dof_count", _i32),
        ("dim", _i32),
        ("dof_coordinates", _p),
        ("cell_count", _i32),
        ("local_dofs", _i32),
        ("cell_dofs", _p),
        ("stiffness", _p),
        ("mass", _p),
        ("parent_cells", _p),
        ("model_cell_count", _i32),
        ("boundary_count", _i32),
        ("boundary_local", _i32),
        ("boundary_dofs", _p),
        ("boundary_cells", _p),
        ("boundary_mass", _p),
        ("boundary_coefficients", _p),
        ("wavenumber_count", _i32),
        ("wavenumbers", _p),
        ("weights", _p),
        ("electrode_count", _i32),
        ("receiver_width", _i32),
        ("receiver_dofs", _p),
        ("receiver_weights", _p),
        ("measurement_count", _i32),
        ("abmn", _p),
        ("source_cell_ptr", _p),
        ("source_cells", _p),
        ("fixed_count", _i32),
        ("fixed_dofs", _p),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("dof_count", _i32),
        ("nnz", _i32),
        ("block_count", _i32),
        ("max_block", _i32),
        ("levels", _i32),
        ("features", _i32),
        ("factor_doubles_per_system", _i64),
        ("contributions", _i64),
    ]


class Tuning(ctypes.Structure):
    """``adt_tuning``: launch shapes of one plan (and, from ``adt_autotune``, their times)."""

    _fields_ = [
        ("strip_fill", _i32),
        ("split_fill", _i32),
        ("jacobian_kernel", _i32),
        ("fields_ms", ctypes.c_float),
        ("jacobian_ms", ctypes.c_float),
    ]

    def as_dict(self) -> dict:
        return {"strip_fill": self.strip_fill, "split_fill": self.split_fill,
                "jacobian_kernel": JACOBIAN_KERNELS[self.jacobian_kernel],
                "fields_ms": float(self.fields_ms), "jacobian_ms": float(self.jacobian_ms)}


_lib = None


def load_library(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load the shared library (once) and declare its signatures."""

    global _lib
    if _lib is not None and path is None:
        return _lib
    target = Path(path) if path is not None else LIBRARY
    if not target.exists():
        raise ImportError(
            f"{target.name} is not built; run __graft_entry__.build() or make -C ad-tlert_b200/csrc"
        )
    lib = ctypes.CDLL(str(target))
    status = ctypes.c_int
    signatures = {
        "adt_plan_create": (status, [ctypes.POINTER(Problem), ctypes.POINTER(_p)]),
        "adt_plan_destroy": (status, [_p]),
        "adt_plan_get_info": (status, [_p, ctypes.POINTER(PlanInfo)]),
        "adt_plan_dof_order": (status, [_p, _p]),
        "adt_last_error": (status, [_p, ctypes.c_char_p, ctypes.c_size_t]),
        "adt_set_primary": (status, [_p, _p, _p]),
        "adt_set_static_rhs": (status, [_p, _p, _p, _p]),
        "adt_factorize": (status, [_p, _i32, _p, _i32, _p]),
        "adt_factorize_fields": (status, [_p, _i32, _p, _i32, _p]),
        "adt_solve_fields": (status, [_p, _i32, _p, _i32, _p, _p]),
        "adt_solve": (status, [_p, _i32, _i32, _i32, _p, _p]),
        "adt_factorize_wavenumbers": (status, [_p, _i32, _p, _i32, _i32, _p]),
        "adt_forward": (status, [_p, _i32, _p, _i32, _p, _p, _p, _p]),
        "adt_jacobian": (status, [_p, _i32, _p, _p, _i32, _i32, _p, _p]),
        "adt_measure": (status, [_p, _p, _i32, _p, _p, _p, _p]),
        "adt_integrated_potentials": (status, [_p, _p, _p, _p]),
        "adt_normal_jacobian": (status, [_p, _p, _i32, _i32, _p, _p]),
        "adt_normal_jacobian_to_host": (status, [_p, _p, _p, _p, _i32, _p]),
        "adt_aggregate_columns": (status, [_p, _i32, _i32, _p, _p, _p, _i32, _i32, _p, _p]),
        "adt_vjp": (status, [_p, _i32, _p, _p, _p, _p, _i32, _p, _p]),
        "adt_adjoint_jacobian": (status, [_p, _i32, _p, _p, _p, _i32, _i32, _i32, _i32, _p, _p]),
        "adt_jvp": (status, [_p, _i32, _p, _p, _p, _p, _p, _p]),
        "adt_normal_vjp": (status, [_p, _p, _p, _i32, _p, _p]),
        "adt_normal_jvp": (status, [_p, _p, _p, _i32, _p, _p]),
        "adt_boundary_jacobian": (status, [_p, _p, _i32, _i32, _p, _p]),
        "adt_measure_static": (status, [_p, _p, _i32, _p, _p, _p]),
        "adt_scale_rows_columns": (status, [_p, _i32, _i32, _p, _p, _p]),
        "adt_fingerprint": (status, [_p, _p, _i64, _i32, _p, _p]),
        "adt_fingerprint_host": (status, [_p, _i64, _i32, _p]),
        "adt_gn_workspace_bytes": (status, [_i32, _i32, _i32, _i32, _p]),
        "adt_gn_step": (status, [_p, _p, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, ctypes.c_double, ctypes.c_double,
                                 _i32, ctypes.c_double, _p, _p, ctypes.c_size_t, _i32, _p]),
        "adt_gn_regularize": (status, [_p, _i32, _i32, _p, _p, _p, ctypes.c_double, ctypes.c_double, _p, _p, _p]),
        "adt_mlp_gemm_splits": (_i32, [_i32, _i32, _i32, _i32]),
        "adt_mlp_gemm": (status, [_p, _p, _i32, _i32, _i32, _i32, _p, ctypes.c_size_t, _p, _p]),
        "adt_mlp_epilogue": (status, [_i32, _p, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p]),
        "adt_mlp_loss": (status, [_p, _p, _i32, _i32, _i32, _p, _p, _p, _p]),
        "adt_mlp_bias_grad": (status, [_p, _i32, _i32, _p, _p]),
        "adt_mlp_adam": (status, [_p, _p, _p, _p, _i64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, ctypes.c_float, _p, _p]),
        "adt_mlp_transpose": (status, [_p, _i32, _i32, _p, _p]),
        "adt_mlp_to_bf16": (status, [_p, _i64, _p, _p]),
        "adt_set_jacobian_wait_limit": (status, [_p, ctypes.c_uint32]),
        "adt_kernel_launches": (_i64, [_p]),
        "adt_autotune": (status, [_p, _i32, _p, _i32, _p, _p, _i32, ctypes.POINTER(Tuning), _p]),
        "adt_get_tuning": (status, [_p, ctypes.POINTER(Tuning)]),
        "adt_set_tuning": (status, [_p, ctypes.POINTER(Tuning)]),
        "adt_jacobian_graph_create": (status, [_p, _i32, _p, _p, _p, _p, _p, _p, ctypes.POINTER(_p)]),
        "adt_graph_launch": (status, [_p, _p]),
        "adt_graph_kernels": (_i64, [_p]),
        "adt_graph_destroy": (status, [_p]),
    }
    for name, (restype, argtypes) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if path is None:
        _lib = lib
    return lib


def last_error(plan) -> str:
    buffer = ctypes.create_string_buffer(1024)
    load_library().adt_last_error(plan, buffer, len(buffer))
    return buffer.value.decode(errors="replace")


def check(status: int, plan, what: str) -> None:
    """Raise the reference's exception type for a non-OK status."""

    if status == ADT_OK:
        return
    message = f"{what}: {last_error(plan)}"
    if status == ADT_INVALID_ARG:
        raise ValueError(message)
    if status in (ADT_NONFINITE, ADT_SOLVER_FAIL):
        raise FloatingPointError(message)
    if status == ADT_OOM:
        raise MemoryError(message)
    raise RuntimeError(message)


def ptr(tensor: torch.Tensor | None):
    return None if tensor is None else ctypes.c_void_p(tensor.data_ptr())


def host_ptr(array):
    return None if array is None else array.ctypes.data_as(ctypes.c_void_p)


def stream_handle(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
