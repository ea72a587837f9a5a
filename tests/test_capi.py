"""CPU-side checks of the drop-in boundary: the C-ABI library loads, exports every
entry point include/uaamg.h declares, and rejects bad input without a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT
from uaamg_b200 import _capi

HEADER = os.path.join(ROOT, "include", "uaamg.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^UAAMG_API[^(]*?\b(uaamg_\w+)\s*\(", txt, re.M)))


def test_header_declares_the_bound_entry_points():
    assert declared() == sorted(_capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (uaamg_\w+)", out))
    assert set(declared()) <= exported


def test_build_targets_sm100a_only():
    from uaamg_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_status_strings_and_defaults():
    lib = _capi.load()
    assert lib.uaamg_status_string(_capi.OK) == b"ok"
    assert lib.uaamg_status_string(_capi.NOT_CONVERGED) == b"not converged"
    assert lib.uaamg_status_string(99) == b"unknown status"
    o = _capi.default_options()
    assert (o.precision, o.tol_mode, o.max_iter, o.tol) == (_capi.FP64, _capi.TOL_ABS, 2000, 1e-6)
    assert (o.replace_every, o.preconditioner, o.warm_start) == (10, 1, 0)


def test_null_and_bad_arguments_are_rejected():
    lib = _capi.load()
    assert lib.uaamg_create(None, 0) == _capi.INVALID_ARG
    h = C.c_void_p()
    assert lib.uaamg_create(C.byref(h), 12345) == _capi.INVALID_ARG
    assert lib.uaamg_destroy(None) == _capi.INVALID_ARG
    assert lib.uaamg_solve(None, None, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_project(None, 1.0, None, None, None, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_project_device(None, 1.0, None, None, None, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_static_pressure(None, None, None, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_set_variable_laplacian(None, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_last_error(None) == b"NULL handle"


def test_python_mirror_fails_loudly_without_library(tmp_path):
    # The product path has no fallback: a missing library is an error.
    with pytest.raises(RuntimeError, match="missing"):
        _capi._lib_saved = _capi._lib
        try:
            _capi._lib = None
            _capi.load(str(tmp_path / "nope.so"))
        finally:
            _capi._lib = _capi._lib_saved


def test_batch_and_server_reject_bad_arguments_without_a_gpu():
    lib = _capi.load()
    assert lib.uaamg_solve_batch(None, 0, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_set_autotune(None, 1) == _capi.INVALID_ARG
    cfg = _capi.ServerConfig()
    lib.uaamg_server_default_config(C.byref(cfg))
    assert (cfg.precision, cfg.tol, cfg.warm_start, cfg.max_active) == (_capi.MIXED, 1e-6, 1, 16)
    assert cfg.hbm_budget_bytes == 150 << 30
    s = C.c_void_p()
    assert lib.uaamg_server_start(None, None) == _capi.INVALID_ARG
    cfg.max_active = 0
    assert lib.uaamg_server_start(C.byref(s), C.byref(cfg)) == _capi.INVALID_ARG
    t = C.c_longlong()
    assert lib.uaamg_server_submit(None, None, C.byref(t)) == _capi.INVALID_ARG
    assert lib.uaamg_server_poll(None, 1, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_server_drain(None) == _capi.INVALID_ARG
    assert lib.uaamg_server_info(None, None, None, None) == _capi.INVALID_ARG
    assert lib.uaamg_server_stop(None) == _capi.INVALID_ARG
