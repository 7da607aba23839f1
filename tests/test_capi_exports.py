"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute call, so no GPU needed)."""
import ctypes
import glob
import os
import re

from gample_b200 import capi
from tests.helpers import ROOT


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:gp_status|void|int|const char\*|unsigned long long)\s+(gp_\w+)\s*\(",
                             text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert len(names) >= 30
    assert "gp_sim_create" in names and "gp_field_solve_poisson" in names


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_functions()) <= set(capi.EXPORTS), set(declared_functions()) - set(capi.EXPORTS)


def test_library_loads_without_gpu_and_reports_errors():
    L = capi.lib()
    assert L.gp_version().startswith(b"gample_b200")
    n = L.gp_device_count()
    assert n >= 0
    # a null handle is an argument error, not a crash
    assert L.gp_sim_run(None, 1) == 1
    assert b"null" in L.gp_last_error()
