"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

from terraneo_b200 import _capi


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(os.path.dirname(_capi.HEADER_PATH), "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"TN_API\s+[\w\s\*]+?\b(tn_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "tn_mesh_create" in syms and "tn_epsdivdiv_apply_f64" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    _capi.lib()
    missing = [s for s in declared_symbols() if s not in _capi._SIGS]
    assert not missing, missing


def test_last_error_without_gpu():
    # tn_last_error is pure host code
    assert isinstance(_capi.lib().tn_last_error(), bytes)
