"""The engine library loads and exports every entry point include/dms.h declares (no GPU call)."""
import ctypes
import os
import re

import pytest

from dms_ctypes import ENGINE_LIB, REPO


def declared_functions():
    src = open(os.path.join(REPO, "include", "dms.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(dms_[a-z_0-9]+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("dms_create", "dms_destroy", "dms_load_solar_model", "dms_add_point", "dms_run", "dms_run_records",
                 "dms_get_results", "dms_rate", "dms_cancel", "dms_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(ENGINE_LIB):
        pytest.skip("libdms_cuda.so not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(ENGINE_LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.dms_num_bins() == 2000
