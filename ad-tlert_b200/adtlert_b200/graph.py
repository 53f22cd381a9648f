"""Fresh-model Jacobians replayed from a captured CUDA graph (``adt_jacobian_graph_create``).

``jacobian()`` enqueues about 35 dependent kernels per model (assembly, the level-by-level
factorization with the field right-hand side, the backward substitution, the measurement and
the Jacobian kernel). For a stream of models through one operator -- time-lapse steps, Monte
Carlo draws, training data for a surrogate -- the chain is captured once and every model costs
one graph launch: ``graph(sigma)`` copies the model into the graph's input buffer and replays,
and returns the Jacobian on the GPU (the graph's own buffer, overwritten by the next call). The
reference has no counterpart (its ``jacobian()`` issues its launches per call,
adtlert/forward/ert2p5d.py:945-1010).
"""

from __future__ import annotations

import ctypes

import torch

from . import _native


class JacobianGraph:
    def __init__(self, operator) -> None:
        self.operator = operator
        device = operator.device
        columns = operator.columns if hasattr(operator, "columns") else operator.E
        self.cells = getattr(operator, "Cd", operator.C)
        self.sigma = torch.ones((operator.C,), dtype=torch.float32, device=device)
        self.fields = torch.empty((1, getattr(operator, "W", 1), operator.N, columns), dtype=torch.float32, device=device)
        self.normal = torch.empty((1, operator.D), dtype=torch.float64, device=device)
        self.reciprocal = torch.empty_like(self.normal)
        self.J = torch.empty((operator.D, self.cells), dtype=torch.float32, device=device)
        self.slot = operator._solver.private()
        self._handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            operator._call("adt_jacobian_graph_create", self.slot, _native.ptr(self.sigma), _native.ptr(self.fields),
                           _native.ptr(self.normal), _native.ptr(self.reciprocal), _native.ptr(self.J),
                           operator._stream(), ctypes.byref(self._handle))
        self.kernels = int(operator._lib.adt_graph_kernels(self._handle))

    def launch(self) -> None:
        """Replay on the current stream with whatever ``self.sigma`` holds."""

        op = self.operator
        _native.check(op._lib.adt_graph_launch(self._handle, op._stream()), op._plan, "adt_graph_launch")

    def __call__(self, conductivity) -> torch.Tensor:
        """J (D, discretization cells) float32 on the GPU of one model (host or device)."""

        sigma = self.operator._sigma(conductivity) if not torch.is_tensor(conductivity) or \
            conductivity.device.type == "cpu" else conductivity
        self.sigma.copy_(sigma.reshape(-1), non_blocking=True)
        self.launch()
        return self.J

    def close(self) -> None:
        if self._handle:
            torch.cuda.current_stream(self.operator.device).synchronize()
            self.operator._lib.adt_graph_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
