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
    d.iorder = 5                                     # beyond the reference's |m| <= 3 rotation tables
    assert lib.fg_stage_create(C.byref(d), 0, C.byref(h)) == _lib.FG_ERR_VALUE
    d.iorder = -1
    assert lib.fg_stage_create(C.byref(d), 0, C.byref(h)) == _lib.FG_ERR_VALUE


def test_new_entry_points_refuse_bad_arguments_on_the_host():
    """The path finder, pair-table, misfit and column entry points check sizes and pointers before any launch."""
    lib = _lib.load()
    V = _lib.FG_ERR_VALUE
    assert lib.fg_pf_candidates(None, 10, 1.0, None, None, 1, 1, 5.0, None, None, None, None, None) == V       # null pos
    assert lib.fg_pf_candidates(None, 10, 1.0, None, None, 1, 0, 5.0, None, None, None, None, None) == V       # per_frame 0
    assert lib.fg_pf_extend(1, 0, None, None, None, None, None, 10.0, None, None, None, None, None, None) == V
    assert lib.fg_pf_extend(1, 9, None, None, None, None, None, 10.0, None, None, None, None, None, None) == V
    assert lib.fg_pf_terminal(-1, 2, None, None, None, None, None, None) == V
    assert lib.fg_pf_describe(1, 10, None, None, None, None, None, None, None, None, None, None, None, None, None, None,
                              None) == V
    assert lib.fg_pair_histogram(None, 1, 4, 0.0, None, None, 0, None, 1, 1.5, 0.01, 1, 5.0, None, None, None) == V   # nr 1
    assert lib.fg_pair_ss_grad(None, 1, 4, 0.0, None, None, 1, None, 1.5, 0.0, 10, 5.0, 1.0, None, None) == V        # dr 0
    assert lib.fg_rspace_misfit(-1, 401, 100, None, None, None, 1.0, None, None, None) == V
    assert lib.fg_rspace_misfit(1, 401, 100, None, None, None, 1.0, None, None, None) == V                  # nulls
    assert lib.fg_path_columns(1, 0, 0, None, None, None, None, None, None) == V                            # E 0
    assert lib.fg_path_columns(1, 60, 7, None, None, None, None, None, None) == V
    assert lib.fg_stage_set_fused_variant(None, 0, 0) == V                                           # null stage
    assert lib.fg_chi_reduce_words(None, 0, None, 401, None, None, None, None, None, None, None, 0, None) == V
    assert lib.fg_rows_from_words(-1, 401, None, None, None) == V
    assert lib.fg_rows_from_words(2, 401, None, None, None) == V                                       # null words
    assert lib.fg_rows_from_words(0, 401, None, None, None) == _lib.FG_OK                              # nothing to do
    assert lib.fg_path_geometry(1, 10, None, None, None, None, None) == V                              # nleg 10
    assert lib.fg_path_geometry_backward(1, 3, None, None, None, None, None, None) == V
    assert lib.fg_stage_set_launch(None, 4, 4) == V
    assert lib.fg_pf_enumerate_one(None, 10, 1.0, None, 0, None, None, 5.0, 3, 0.0, 1, None, None, None, None) == V
    assert lib.fg_pf_result_gather(None, 2, None, None, None, None, None, None) == V
    lib.fg_pf_result_destroy(None)                                                                      # a no-op
    cost = (C.c_double * 4)(3.0, 1.0, 2.0, 2.0)
    owner = (C.c_int32 * 4)()
    assert lib.fg_shard_lpt(cost, 4, 0, owner) == V                                                    # no ranks
    assert lib.fg_shard_lpt(cost, 4, 2, owner) == _lib.FG_OK
    assert sorted(sum(cost[i] for i in range(4) if owner[i] == r) for r in range(2)) == [4.0, 4.0]
    w = (C.c_int64 * 3)()
    sl = (C.c_float * 3)(1.0, 1.0005, 1.5)
    off = (C.c_int64 * 2)(0, 3)
    assert lib.fg_pf_windows(sl, off, 1, C.c_float(1e-3), w) == _lib.FG_OK
    assert list(w) == [0, 0, 1]


def test_fused_entry_points_refuse_batches_without_their_arrays():
    """A batch whose per-path arrays are missing, or that has paths but no rows, is refused before any launch (the
    stage handle is not read: the batch is checked first), so no kernel ever reads through a null device pointer."""
    lib = _lib.load()
    V = _lib.FG_ERR_VALUE
    fake_stage = C.create_string_buffer(64)          # never dereferenced: the batch check fails first
    dummy = C.create_string_buffer(64)

    def paths(n, nrows, order=True, row=True, nleg_max=3):
        a = C.addressof(dummy)
        return _lib.Paths(n, nleg_max, nrows, a, a, a, a, None, a if row else None, a if order else None)

    bad = [paths(5, 1, order=False), paths(5, 1, row=False), paths(5, 0), paths(-1, 1), paths(5, 1, nleg_max=10)]
    for ps in bad:
        assert lib.fg_chi_reduce(fake_stage, 0, C.byref(ps), 401, None, None, None, None, None, None, None, 0,
                                 None) == V
        assert lib.fg_chi_reduce_noalloc(fake_stage, 0, C.byref(ps), 401, None, None, None, None, None) == V
        assert lib.fg_chi_reduce_backward(fake_stage, 0, C.byref(ps), 401, None, None, None, None, None, None, None,
                                          None, None, None, 0, None) == V
    with pytest.raises(ValueError, match="null array"):
        _lib.check(lib.fg_chi_reduce(fake_stage, 0, C.byref(bad[0]), 401, None, None, None, None, None, None, None,
                                     0, None))


def test_potential_index_errors_raise_index_error():
    """The library's out-of-range potential report maps to the reference's exception for a bad table index."""
    _lib.load()
    import feffgpu_b200._lib as L
    orig = L._lib.fg_last_error
    try:
        L._lib.fg_last_error = lambda: b"potential index outside 0..nph (the rows are NaN)"
        with pytest.raises(IndexError):
            L.check(L.FG_ERR_VALUE)
    finally:
        L._lib.fg_last_error = orig
