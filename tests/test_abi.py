"""The C-ABI library loads without a GPU and exports every entry point include/sgipc.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "sgipc.h")).read()
    return sorted(set(re.findall(r"^(?:SgipcStatus|const char\*)\s+(sgipc_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "sgipc_create" in names and "sgipc_pcg_solve" in names and len(names) >= 18


def test_library_exports_every_declared_symbol():
    from sgipc import _native

    lib = ctypes.CDLL(_native.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
    # the Python binding covers the same set
    assert set(declared_functions()) == set(_native.SIGNATURES)


def test_binding_loads_and_reports_bad_input_without_gpu():
    from sgipc import _native as N

    L = N.lib()
    assert L.sgipc_status_string(N.BAD_INPUT) == b"bad input"
    h = ctypes.c_void_p()
    # a null topology is rejected before any CUDA call
    assert L.sgipc_create(None, 0, ctypes.byref(h)) == N.BAD_INPUT
    t = N.SgipcTopology()
    t.vertex_num = -1
    assert L.sgipc_create(ctypes.byref(t), 0, ctypes.byref(h)) == N.BAD_INPUT
