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


def test_backend_methods_mirror_the_reference_table():
    """bbhx_b200.backend binds exactly BBHx's backend methods (the fields of
    BBHxBackendMethods, src/bbhx/cutils/__init__.py:13-23) with the positional arity of the
    reference's Cython wrappers, each onto a declared entry point."""
    import numpy as np
    import pytest

    from bbhx_b200 import backend

    reference_fields = {"hdyn_wrap", "direct_like_wrap", "direct_sum_wrap", "InterpTDI_wrap",
                        "pyFastLISAResponse", "waveform_amp_phase_wrap",
                        "get_phenomhm_ringdown_frequencies", "get_phenomd_ringdown_frequencies",
                        "interpolate_wrap"}
    assert set(backend.METHOD_NAMES) == reference_fields
    arity = {"waveform_amp_phase_wrap": 16, "get_phenomhm_ringdown_frequencies": 10,
             "get_phenomd_ringdown_frequencies": 16, "interpolate_wrap": 10, "InterpTDI_wrap": 16,
             "direct_sum_wrap": 8, "direct_like_wrap": 9, "hdyn_wrap": 8}
    declared = set(declared_functions())
    for name, (cname, slots) in backend._METHODS.items():
        assert len(slots) == arity[name], name
        assert cname in declared, cname
    assert len(backend._RESPONSE_SLOTS) == 17  # LISA_response_wrap (lisaresponse.pyx:78-121)
    # host memory in a device slot is refused before anything reaches the library's kernels
    with pytest.raises(TypeError, match="device memory"):
        backend._device_addr(np.zeros(4), "f8", "x")


def test_workspace_registration_rules():
    """bbhx_workspace_set needs no GPU: it records the caller's buffer for the calling thread.
    A 256-byte aligned base is taken, an unaligned one or a tiny size is refused (status 1), a
    null base returns to the stream-ordered pool, and nothing has been needed yet (peak 0)."""
    from bbhx_b200 import build_ext

    build_ext.build()
    lib = ctypes.CDLL(build_ext.OUT)
    lib.bbhx_workspace_set.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    lib.bbhx_workspace_peak.restype = ctypes.c_size_t
    assert lib.bbhx_workspace_set(ctypes.c_void_p(1 << 20), 1 << 16) == 0
    assert lib.bbhx_workspace_peak() == 0
    assert lib.bbhx_workspace_set(ctypes.c_void_p((1 << 20) + 8), 1 << 16) == 1
    assert lib.bbhx_workspace_set(ctypes.c_void_p(1 << 20), 16) == 1
    assert lib.bbhx_workspace_set(ctypes.c_void_p(0), 0) == 0


def test_descriptor_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the C descriptor structs (bbhx_b200.uneven) have the header's
    sizes and field offsets (checked with the host C compiler on the header itself)."""
    import shutil
    import subprocess

    import pytest

    from bbhx_b200.uneven import DirectGroupC, DirectSourceC, HdynGroupC, HdynSourceC

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    mirrors = {"bbhx_direct_group": DirectGroupC, "bbhx_hdyn_group": HdynGroupC,
               "bbhx_direct_source": DirectSourceC, "bbhx_hdyn_source": HdynSourceC}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "bbhx_b200.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out if ln.strip()}
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_misaligned_record_buffer_is_refused():
    """bbhx_phenomhm_setup writes its records with 16-byte stores: a buffer that is not 16-byte
    aligned is refused with status 1 before anything is launched (no GPU needed)."""
    from bbhx_b200 import build_ext

    build_ext.build()
    lib = ctypes.CDLL(build_ext.OUT)
    f = lib.bbhx_phenomhm_setup
    f.argtypes = [ctypes.c_void_p] * 10 + [ctypes.c_int] * 3 + [ctypes.c_void_p]
    f.restype = ctypes.c_int
    args = [None] * 9 + [6, 1, 0, None]
    assert f(ctypes.c_void_p((1 << 20) + 8), *args) == 1
    lib.bbhx_last_error_string.restype = ctypes.c_char_p
    assert b"aligned" in lib.bbhx_last_error_string()
