"""The C-ABI library loads and exports every entry point include/bbhx_b200.h declares
(no GPU needed: nothing is called except symbol lookup)."""
import ctypes
import os
import re

from conftest import REPO


def declared_functions():
    src = open(os.path.join(REPO, "include", "bbhx_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bbhx_[a-zA-Z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "bbhx_waveform_amp_phase" in names
    assert "bbhx_direct_like_fused" in names
    assert len(names) >= 25


def test_library_exports_all_declared_symbols():
    from bbhx_b200 import build_ext

    build_ext.build()
    lib = ctypes.CDLL(build_ext.OUT)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from bbhx_b200 import _lib

    bound = set(_lib.exported_symbols())
    missing = [n for n in declared_functions() if n not in bound]
    assert not missing, missing
