"""LRU of solved fields keyed by a hash of the model, and the batching of cache misses
(semantics of adtlert/forward/field_cache.py:17-110)."""

from __future__ import annotations

import hashlib
from collections import OrderedDict
from collections.abc import Callable, Sequence

import numpy as np
import torch


def step_batches(steps: Sequence[int], batch_steps: int) -> list[list[int]]:
    """Near-equal consecutive batches of at most ``batch_steps`` steps."""

    steps = list(steps)
    if not steps:
        return []
    if len(steps) <= batch_steps:
        return [[int(step) for step in steps]]
    count = -(-len(steps) // batch_steps)
    return [list(map(int, batch)) for batch in np.array_split(np.asarray(steps), count)]


def newest_batches_first(step_count: int, batch_steps: int) -> list[list[int]]:
    """Forward batches in reverse, so an adjoint pass starts with the factorization still held."""

    return step_batches(range(step_count), batch_steps)[::-1]


def factorization_name(keys) -> tuple | None:
    """Name of a batch's factorized operators, or ``None`` when any model is uncached."""

    named = tuple(key for key in keys if key is not None)
    return named if len(named) == len(keys) else None


class FieldCache:
    """Fields of recently solved models keyed by a digest of the model bytes (SHA-256, the
    fastest of hashlib's digests on the host here, truncated to 16 bytes) and their dtype."""

    def __init__(self, max_entries: int) -> None:
        if int(max_entries) < 0:
            raise ValueError("normal_field_cache_max_entries must be non-negative")
        self.max_entries = int(max_entries)
        self._entries: OrderedDict = OrderedDict()
        self.hits = self.misses = 0

    def key(self, model: torch.Tensor):
        if self.max_entries < 1:
            return None
        host = np.ascontiguousarray(model.detach().cpu().numpy())
        return hashlib.sha256(host.view(np.uint8)).digest()[:16] + host.dtype.str.encode()

    def _lookup(self, key):
        if key is None:
            return None
        found = self._entries.get(key)
        if found is None:
            self.misses += 1
        else:
            self.hits += 1
            self._entries.move_to_end(key)
        return found

    def _store(self, key, fields) -> None:
        if key is None:
            return
        self._entries[key] = fields
        self._entries.move_to_end(key)
        while len(self._entries) > self.max_entries:
            self._entries.popitem(last=False)

    def solve_series(self, models: torch.Tensor, batch_steps: int, solve: Callable):
        keys = [self.key(model) for model in models]
        fields = {}
        for step, key in enumerate(keys):
            found = self._lookup(key)
            if found is not None:
                fields[step] = found
        missing = [step for step in range(len(keys)) if step not in fields]
        for batch in step_batches(missing, batch_steps):
            name = factorization_name([keys[step] for step in batch])
            chosen = models if batch == list(range(len(models))) else models[batch]
            for step, solved in zip(batch, solve(chosen, name), strict=True):
                fields[step] = solved
                self._store(keys[step], solved)
        return [fields[step] for step in range(len(keys))], keys

    def clear(self) -> None:
        self._entries.clear()

    def info(self) -> dict[str, int]:
        return {"entries": len(self._entries), "max_entries": self.max_entries, "hits": self.hits, "misses": self.misses}
