"""The field store on CPU: batching, the LRU contract the reference's operators expose
(adtlert/forward/field_cache.py:17-110), and the host fingerprint of the library."""

import ctypes

import numpy as np
import pytest
import torch

from adtlert_b200 import _native
from adtlert_b200.field_store import FieldStore, adjoint_batches, batch_name, even_batches, model_fingerprints


def test_even_batches_match_near_equal_consecutive_splits():
    for count in range(0, 40):
        for limit in range(1, 12):
            items = list(range(100, 100 + count))
            runs = even_batches(items, limit)
            assert [i for run in runs for i in run] == items
            if count:
                assert len(runs) == -(-count // limit)
                sizes = [len(r) for r in runs]
                assert max(sizes) <= limit and max(sizes) - min(sizes) <= 1
                assert sizes == sorted(sizes, reverse=True)
                # the same partition as numpy's array_split, which the reference uses
                assert runs == [list(map(int, part)) for part in np.array_split(np.asarray(items), len(runs))]
    assert adjoint_batches(5, 2) == [[4], [2, 3], [0, 1]]


def test_batch_names():
    assert batch_name([b"a", b"b"]) == (b"a", b"b")
    assert batch_name([b"a", None]) is None


def _store(capacity):
    return FieldStore(capacity, lambda models: [m.numpy().tobytes() for m in models])


def test_lru_hits_misses_and_batches():
    store = _store(3)
    solved = []

    def solve(models, name):
        solved.append((models.shape[0], name is not None))
        return [f"f{float(m[0])}" for m in models]

    series = torch.arange(5, dtype=torch.float32)[:, None].repeat(1, 4)
    fields, keys = store.fields(series, 2, solve)
    assert fields == [f"f{i}.0" for i in range(5)] and len(keys) == 5
    assert solved == [(2, True), (2, True), (1, True)]
    assert store.info() == {"entries": 3, "max_entries": 3, "hits": 0, "misses": 5}
    solved.clear()
    fields, _ = store.fields(series[[4, 0]], 8, solve)  # 4 is remembered, 0 was evicted
    assert fields == ["f4.0", "f0.0"] and solved == [(1, True)]
    assert store.info()["hits"] == 1 and store.info()["misses"] == 6
    store.clear()
    assert store.info()["entries"] == 0


def test_capacity_zero_remembers_nothing_and_names_nothing():
    store = _store(0)
    names = []
    store.fields(torch.ones((3, 2)), 8, lambda m, name: names.append(name) or [None] * len(m))
    store.fields(torch.ones((3, 2)), 8, lambda m, name: names.append(name) or [None] * len(m))
    assert names == [None, None]
    assert store.info() == {"entries": 0, "max_entries": 0, "hits": 0, "misses": 0}
    with pytest.raises(ValueError, match="normal_field_cache_max_entries must be non-negative"):
        _store(-1)


def test_host_fingerprint_keys():
    lib = _native.load_library()
    rng = np.random.default_rng(0)
    models = torch.as_tensor(rng.uniform(0.001, 1.0, (6, 9600)), dtype=torch.float32)
    keys = model_fingerprints(lib, None, models, None)
    assert len(set(keys)) == 6 and all(len(k) == 16 + len(b"torch.float32") for k in keys)
    assert model_fingerprints(lib, None, models.clone(), None) == keys  # content, not identity
    flipped = models.clone()
    flipped[3, 4711] = float(np.nextafter(np.float32(flipped[3, 4711]), np.float32(2.0)))
    changed = model_fingerprints(lib, None, flipped, None)
    assert changed[3] != keys[3] and changed[:3] == keys[:3] and changed[4:] == keys[4:]
    swapped = models.clone()
    swapped[0, [10, 11]] = swapped[0, [11, 10]]  # position matters
    assert model_fingerprints(lib, None, swapped, None)[0] != keys[0]
    wide = model_fingerprints(lib, None, models.double(), None)
    assert wide[0] != keys[0] and wide[0].endswith(b"torch.float64")
    out = np.zeros(2, dtype=np.uint64)
    assert lib.adt_fingerprint_host(ctypes.c_void_p(models.data_ptr()), 6, 1,
                                    _native.host_ptr(out)) == _native.ADT_INVALID_ARG  # not whole words
