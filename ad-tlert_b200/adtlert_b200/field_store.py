"""Solved fields of recent models, found again by a content fingerprint of the model.

The operators expose, and the reference's tests count, this behaviour of its field cache
(adtlert/forward/field_cache.py:17-110): at most ``capacity`` models are remembered and the
least recently used one leaves first; a capacity of 0 remembers nothing and names no
factorization; every lookup of a keyed model counts as a hit or a miss; the models of a series
that are not remembered are solved together in consecutive batches of near-equal size, at most
``batch_steps`` models each, and each batch's factorization is named by its models' keys (no
name when any model is unkeyed), so a solver slot that holds that name is reused.

Where the key comes from is this library's own: the solved fields live on the GPU and the
models often do too, so a model is keyed by a 128-bit content fingerprint computed where it
lies (``adt_fingerprint``: one kernel launch for a whole series, 16 bytes per model read back,
instead of copying every model to the host to hash it; ``adt_fingerprint_host``, the same
function on the host, for models in host memory). Equal values of the same dtype give the same
key on either device.
"""

from __future__ import annotations

from collections import OrderedDict
from collections.abc import Callable, Sequence

import numpy as np
import torch

from . import _native

Tensor = torch.Tensor
Key = bytes | None


def even_batches(items: Sequence[int], limit: int) -> list[list[int]]:
    """``items`` cut into as few consecutive runs as a limit of ``limit`` per run allows, whose
    lengths differ by at most one (the longer runs first)."""

    items = [int(item) for item in items]
    if not items:
        return []
    runs = -(-len(items) // int(limit))
    short, longer = divmod(len(items), runs)
    out, start = [], 0
    for run in range(runs):
        stop = start + short + (1 if run < longer else 0)
        out.append(items[start:stop])
        start = stop
    return out


def adjoint_batches(count: int, limit: int) -> list[list[int]]:
    """The forward batches of ``count`` steps, last batch first: an adjoint pass over a series
    then starts with the factorization the solver still holds."""

    return even_batches(range(count), limit)[::-1]


def batch_name(keys: Sequence[Key]) -> tuple[bytes, ...] | None:
    """Name of a batch's factorization: its models' keys, or None when one model is unkeyed."""

    return None if any(key is None for key in keys) else tuple(keys)


_MAX_MODELS_PER_LAUNCH = 65535


def model_fingerprints(lib, plan, models: Tensor, stream) -> list[bytes]:
    """Content keys of the rows of ``models`` (S, cells): fingerprint bytes + dtype tag."""

    models = models.detach().contiguous()
    count = int(models.shape[0])
    row_bytes = int(models.shape[1]) * models.element_size()
    tag = str(models.dtype).encode()
    if models.is_cuda:
        words = torch.empty((count, 2), dtype=torch.int64, device=models.device)
        for start in range(0, count, _MAX_MODELS_PER_LAUNCH):
            rows = min(_MAX_MODELS_PER_LAUNCH, count - start)
            _native.check(lib.adt_fingerprint(plan, _native.ptr(models[start]), row_bytes, rows,
                                              _native.ptr(words[start]), stream), plan, "adt_fingerprint")
        host = words.cpu().numpy()
    else:
        host = np.empty((count, 2), dtype=np.int64)
        for start in range(0, count, _MAX_MODELS_PER_LAUNCH):
            rows = min(_MAX_MODELS_PER_LAUNCH, count - start)
            status = lib.adt_fingerprint_host(models[start].data_ptr(), row_bytes, rows, _native.host_ptr(host[start:]))
            _native.check(status, None, "adt_fingerprint_host")
    return [host[row].tobytes() + tag for row in range(count)]


class FieldStore:
    """Least-recently-used map from model keys to solved fields."""

    def __init__(self, capacity: int, fingerprint: Callable[[Tensor], list[bytes]]) -> None:
        if int(capacity) < 0:
            raise ValueError("normal_field_cache_max_entries must be non-negative")
        self.capacity = int(capacity)
        self._fingerprint = fingerprint
        self._recent: OrderedDict[bytes, object] = OrderedDict()
        self.hits = 0
        self.misses = 0

    def keys(self, models: Tensor) -> list[Key]:
        """Keys of the rows of ``models`` (all None when nothing is remembered)."""

        if self.capacity == 0:
            return [None] * int(models.shape[0])
        return self._fingerprint(models)

    def key(self, model: Tensor) -> Key:
        return self.keys(model[None])[0]

    def _recall(self, key: Key):
        if key is None:
            return None
        fields = self._recent.pop(key, None)
        if fields is None:
            self.misses += 1
            return None
        self.hits += 1
        self._recent[key] = fields  # now the most recent
        return fields

    def _remember(self, key: Key, fields) -> None:
        if key is None:
            return
        self._recent.pop(key, None)
        self._recent[key] = fields
        while len(self._recent) > self.capacity:
            self._recent.popitem(last=False)

    def fields(self, models: Tensor, batch_steps: int, solve: Callable) -> tuple[list, list[Key]]:
        """Fields of every row of ``models`` and the rows' keys; rows not remembered are solved by
        ``solve(batch_models, batch_name)``, which returns one fields object per row."""

        keys = self.keys(models)
        found = [self._recall(key) for key in keys]
        unsolved = [row for row, fields in enumerate(found) if fields is None]
        for batch in even_batches(unsolved, batch_steps):
            chosen = models if len(batch) == len(found) else models[batch]
            for row, fields in zip(batch, solve(chosen, batch_name([keys[row] for row in batch])), strict=True):
                found[row] = fields
                self._remember(keys[row], fields)
        return found, keys

    def clear(self) -> None:
        self._recent.clear()

    def info(self) -> dict[str, int]:
        return {"entries": len(self._recent), "max_entries": self.capacity, "hits": self.hits, "misses": self.misses}
