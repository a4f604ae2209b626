"""The C-ABI library: it loads, exports every entry point that include/feffgpu_b200.h declares, and reports argument
errors without touching a GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

from feffgpu_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "feffgpu_b200.h"


def declared():
    return sorted(set(re.findall(r"FG_API\s+[\w\s\*]+?\b(fg_\w+)\s*\(", HEADER.read_text())))


def test_header_and_binding_agree():
    assert declared() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared():
        assert hasattr(lib, name), name


def test_argument_errors_map_to_exceptions():
    lib = _lib.load()
    rc = lib.fg_cchi(None, 0, 1, 3, None, 0, None, None, None, None, None)
    assert rc == _lib.FG_ERR_VALUE
    with pytest.raises(ValueError, match="null stage"):
        _lib.check(rc)
    assert lib.fg_set_launch(9, 0) == _lib.FG_ERR_VALUE
    assert lib.fg_set_launch(0, 0) == _lib.FG_OK


def test_stage_create_rejects_spin_and_iorder():
    lib = _lib.load()
    d = _lib.PhaseDesc()
    d.nsp = 2
    h = C.c_void_p()
    rc = lib.fg_stage_create(C.byref(d), 0, C.byref(h))
    assert rc == _lib.FG_ERR_NOT_IMPLEMENTED
    d.nsp, d.iorder = 1, 12
    assert lib.fg_stage_create(C.byref(d), 0, C.byref(h)) == _lib.FG_ERR_NOT_IMPLEMENTED
