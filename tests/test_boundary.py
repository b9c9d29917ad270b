"""C ABI boundary checks that need no GPU: the library loads, exports every
function include/gospl_b200.h declares, and the stats struct matches."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "gospl_b200.h")).read()
    return sorted(set(re.findall(r"\b(gs_[a-z_0-9]+)\s*\(", src)))


def test_library_builds_and_loads():
    from gospl_b200 import build as B
    B.build()
    from gospl_b200 import _lib
    L = _lib.load()
    assert L.gs_version() >= 100


def test_exports_every_declared_symbol():
    from gospl_b200 import _lib
    L = _lib.load()
    names = _declared()
    assert len(names) >= 12
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(_lib.EXPORTS)


def test_every_export_has_argument_types():
    """ctypes cannot pass Python floats without declared argument types: every
    entry point with arguments declares them."""
    from gospl_b200 import _lib
    L = _lib.load()
    for name in _lib.EXPORTS:
        if name in ("gs_version",):
            continue
        assert getattr(L, name).argtypes is not None, name


def test_sed_change_rejects_null_plan():
    from gospl_b200 import _lib
    L = _lib.load()
    st = _lib.GsStats()
    assert L.gs_sed_change(None, None, None, None, None, 0.0, -6000.0, 1.0, 1e9, 100.0, None, None, None, None,
                           None, None, None, None, ctypes.byref(st)) == 1


def test_stats_struct_layout():
    from gospl_b200 import _lib
    assert ctypes.sizeof(_lib.GsStats) == 8 * 4 + 8


def test_null_plan_is_rejected():
    from gospl_b200 import _lib
    L = _lib.load()
    assert L.gs_mfdreceivers(None, 3, 1.1, None, 0.0, None, None, None, None) == 1
    buf = ctypes.create_string_buffer(256)
    assert L.gs_last_error(buf, 256) == 1
    assert b"plan" in buf.value


def test_bad_plan_arguments_are_rejected():
    from gospl_b200 import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.gs_plan_create(-1, None, None, None, None, None, None, None, 0, None, 0, 0, 3,
                            ctypes.byref(h)) == 1
    assert L.gs_plan_create(10, None, None, None, None, None, None, None, 0, None, 0, 0, 13,
                            ctypes.byref(h)) == 1


def test_knob_numbers_used_from_python_match_the_header():
    """The GS_TUNE_* numbers that the Python side and the tests pass to
    gs_plan_tune are the header's."""
    src = open(os.path.join(ROOT, "include", "gospl_b200.h")).read()
    header = {k: int(v) for k, v in re.findall(r"#define (GS_TUNE_[A-Z_]+) (\d+)", src)}
    assert header["GS_TUNE_WARM_START"] == 8
    from gospl_b200 import adjoint
    assert adjoint.GS_TUNE_WARM_START == header["GS_TUNE_WARM_START"]
    import test_gpu_failures
    import test_gpu_warm_start
    assert test_gpu_failures.GS_TUNE_SWEEP_BUDGET == header["GS_TUNE_SWEEP_BUDGET"]
    assert test_gpu_warm_start.GS_TUNE_WARM_START == header["GS_TUNE_WARM_START"]
