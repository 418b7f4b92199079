"""The drop-in boundary: the C-ABI library loads and exports every entry point that
include/qsb200.h declares (no GPU work here)."""
import ctypes
import os
import re

import quichotte_b200 as qb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qsh?_[a-z0-9_]+)\s*\(", text)))


def test_cuda_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(qb.LIB_PATH)
    names = declared("qsb200.h")
    assert len(names) >= 16
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(qb.C_ABI) <= set(names)


def test_host_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(qb.HOST_PATH)
    names = [n for n in declared("qs_host.h") if n.startswith("qsh_")]
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_program_binary_is_built():
    assert os.access(qb.PROGRAM, os.X_OK)
