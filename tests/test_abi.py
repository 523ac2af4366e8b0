"""The C ABI library loads and exports every entry point include/ltg.h declares."""
import os
import re

from libtensor_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "ltg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ltg_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_header_symbols():
    L = _capi.lib()
    missing = [s for s in header_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(header_symbols()) <= set(_capi.declared_symbols())


def test_version_and_error_string():
    L = _capi.lib()
    assert L.ltg_version() >= 100
    assert isinstance(L.ltg_last_error(), bytes)
