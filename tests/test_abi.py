"""The C-ABI library loads without a GPU and exports every entry point its header declares;
argument validation happens before any device call."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pfsht_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(pfsht_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for n in ("pfsht_plan_create", "pfsht_plan_destroy", "pfsht_forward", "pfsht_adjoint",
              "pfsht_ring_work", "pfsht_plan_get_info", "pfsht_workspace_bytes",
              "pfsht_last_error", "pfsht_forward_host", "pfsht_adjoint_host",
              "pfsht_ring_forward", "pfsht_ring_adjoint", "pfsht_nufft_create",
              "pfsht_nufft_exec", "pfsht_nufft_destroy", "pfsht_dfs_double", "pfsht_dfs_fold"):
        assert n in names, n


def test_library_exports_every_declared_symbol(pf):
    lib = C.CDLL(pf._lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(pf):
    assert set(declared_functions()) <= set(pf._lib.SIGNATURES)


def test_version_and_errors_without_device(pf):
    assert "sm_100a" in pf.version()
    lib = pf._lib.load()
    h = C.c_void_p()
    th = np.zeros(4)
    # validation precedes any device call: bad sizes come back as ArgumentError codes
    st = lib.pfsht_plan_create(th.ctypes.data, th.ctypes.data, 4, -1, 1, 1e-8, 0, None, C.byref(h))
    assert st == pf._lib.ERR_ARGUMENT
    assert "lmax" in pf._lib.last_error()
    st = lib.pfsht_plan_create(th.ctypes.data, th.ctypes.data, 4, 8, 0, 1e-8, 0, None, C.byref(h))
    assert st == pf._lib.ERR_ARGUMENT
    st = lib.pfsht_plan_create(th.ctypes.data, th.ctypes.data, 4, 8, 1, 2.0, 0, None, C.byref(h))
    assert st == pf._lib.ERR_ARGUMENT
    st = lib.pfsht_plan_create(None, th.ctypes.data, 4, 8, 1, 1e-8, 0, None, C.byref(h))
    assert st == pf._lib.ERR_ARGUMENT
    st = lib.pfsht_nufft_create(3, 8, 8, 1, 1, 1e-8, th.ctypes.data, th.ctypes.data, 4, C.byref(h))
    assert st == pf._lib.ERR_ARGUMENT


def test_stage_names(pf):
    lib = pf._lib.load()
    n = lib.pfsht_num_stages()
    names = [lib.pfsht_stage_name(i).decode() for i in range(n)]
    assert "ring_fwd" in names and "spread" in names and "interp" in names
    assert lib.pfsht_stage_name(n).decode() == ""


def test_oracle_library_loads(O):
    assert O.next_smooth_even(135) == 144
