"""The C-ABI library loads without a GPU, exports every symbol the headers
declare, and its host-side entry points validate their arguments."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, header)).read()
    return sorted(set(re.findall(r"CPS_API\s+[\w\s\*]*?\b(cps_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    import cpsfdtd_b200 as cps
    names = declared("include/cps_capi.h")
    assert len(names) >= 50
    L = C.CDLL(cps.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_oracle_library_exports_its_header(oracle_mod):
    text = open(os.path.join(ROOT, "oracle", "oracle.h")).read()
    names = sorted(set(re.findall(r"\b(orc2?d?_\w+)\s*\(", text)))
    L = oracle_mod.lib()
    assert all(hasattr(L, n) for n in names)


def test_host_entry_points_reject_bad_arguments():
    import cpsfdtd_b200 as cps
    L = cps.lib()
    ids = np.zeros((5, 5, 5), np.uint8)
    assert L.cps_mesh_rasterize(1, 4, 4, 1e-8, 1e-8, 1e-8, 0, None, ids.ctypes.data, 0) == 1
    assert b"invalid" in L.cps_last_error()
    cnt = C.c_int32(0)
    assert L.cps_port_points_plain(10, 10, 10, 1e-8, 1e-8, 1e-8, b"q", 0.0, 0.0, 0.0, 0.0, 0.0, C.byref(cnt), None) == 1
    assert L.cps_port_points_plain(10, 10, 10, 1e-8, 1e-8, 1e-8, b"x", 5e-8, 0.0, 20e-8, 0.0, 1e-8,
                                   C.byref(cnt), None) == 1  # w2 beyond ny
    assert L.cps_grid_create(None, None) == 1
    assert abs(L.cps_courant_dt(1e-8, 1e-8, 1e-8) - 0.99 / (2.99792458e8 * np.sqrt(3e16))) < 1e-30


def test_grid_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import cpsfdtd_b200 as cps
    with pytest.raises(cps.CpsError):
        cps.Grid(8, 8, 8, 1e-8, 1e-8, 1e-8)


def test_python_status_codes_match_the_header():
    import cpsfdtd_b200 as cps
    text = open(os.path.join(ROOT, "include", "cps_capi.h")).read()
    codes = dict(re.findall(r"\b(CPS_(?:OK|E_\w+))\s*=\s*(\d+)", text))
    assert len(codes) == 10
    for name, v in codes.items():
        assert getattr(cps, name) == int(v), name


def test_recorder_entry_points_validate_without_a_device():
    import cpsfdtd_b200 as cps
    L = cps.lib()
    assert L.cps_grid_set_record(None, 1) == cps.CPS_E_INVALID
    assert L.cps_grid_record_stats(None, None, None, None) == cps.CPS_E_INVALID
    assert L.cps_op_h_bulk(None) == cps.CPS_E_INVALID
