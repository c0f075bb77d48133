"""The C-ABI library loads without a GPU and exports exactly what include/paracfd_b200.h declares;
the Python binding table agrees with the header.  No compute calls."""
import ctypes as C
import os
import re

import pytest

from paracfd_b200 import capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "paracfd_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pcfd_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "pcfd_core_step" in names and "pcfd_pressure_solve_host" in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_matches_header():
    assert sorted(capi.SIGNATURES) == declared_functions()


def test_version_and_error_message_without_gpu():
    lib = capi.load()
    lib.pcfd_version.restype = C.c_char_p
    assert lib.pcfd_version()
    lib.pcfd_last_error_message.restype = C.c_char_p
    lib.pcfd_last_error_message()


def test_null_system_is_rejected_without_gpu():
    lib = capi.load()
    n = C.c_int64()
    assert lib.pcfd_launch_count(None, C.byref(n)) == capi.PCFD_INVALID_ARG
