"""The C ABI: the library loads without a GPU and exports every entry point the header declares."""

import ctypes
import re

import pytest

from adtlert_b200 import _native
from conftest import ROOT

HEADER = ROOT / "include" / "adtlert_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:adt_status|int64_t|int32_t)\s+(adt_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_binding_symbols():
    assert declared_symbols() == sorted(_native.SYMBOLS)


def test_library_exports_every_declared_symbol():
    if not _native.LIBRARY.exists():
        pytest.fail("libadtlert_b200.so is not built (run __graft_entry__.build())")
    lib = _native.load_library()
    for name in declared_symbols():
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr), name


def test_struct_layouts_match_the_header():
    # field order and count of adt_problem / adt_plan_info as declared in the header
    text = HEADER.read_text()
    body = text[text.index("typedef struct {", text.index("adt_stream;")):text.index("} adt_problem;")]
    names = re.findall(r"(\w+);", re.sub(r"/\*.*?\*/", "", body, flags=re.S))
    assert names == [f[0] for f in _native.Problem._fields_]
    assert ctypes.sizeof(_native.PlanInfo) == 5 * 4 + 4 + 2 * 8


def test_invalid_problem_is_rejected_without_a_gpu():
    lib = _native.load_library()
    plan = ctypes.c_void_p()
    status = lib.adt_plan_create(None, ctypes.byref(plan))
    assert status == _native.ADT_INVALID_ARG
    assert "null" in _native.last_error(None)
