"""C ABI surface checks that need no GPU: the library loads and exports every
entry point include/ra_engine.h declares."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ra_engine.h")
LIB = os.path.join(ROOT, "parallel-ra_b200", "libra_b200.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*|void)\s+(ra_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ra_program_execute" in names and "ra_relation_dump_full" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the engine first (python parallel-ra_b200/build.py)"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_all_exports():
    import parallel_ra_b200 as P
    assert set(P.engine.EXPORTS) == set(declared_functions())


def test_status_strings_without_gpu():
    lib = ctypes.CDLL(LIB)
    lib.ra_status_string.restype = ctypes.c_char_p
    assert lib.ra_status_string(0) == b"ok"
    assert lib.ra_status_string(5) == b"unsupported program shape"
    lib.ra_last_error.restype = ctypes.c_char_p
    lib.ra_last_error.argtypes = [ctypes.c_void_p]
    assert lib.ra_last_error(None) == b"null program"


def test_program_create_rejects_bad_device():
    lib = ctypes.CDLL(LIB)
    h = ctypes.c_void_p()
    assert lib.ra_program_create(-1, ctypes.byref(h)) != 0
    assert not h.value
