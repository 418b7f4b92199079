"""The drop-in boundary: the C-ABI library loads and exports every entry point that
include/qsb200.h declares (no GPU work here)."""
import ctypes
import os
import re

import pytest

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


def test_memory_estimate_grows_with_the_problem_and_needs_no_device():
    def helix(ions, turns, delta):
        return qb.Model.helix(N_ions=ions, N_turns=turns, hel_length=0.34 * turns, hel_radius=0.7, hand=1.0,
                              E_CC=0.0, t_hop=1.0, lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5,
                              T=300.0, mu=0.0, dw=1.0, up=1.0, delta=delta, order=2)
    small, wide, long_ = helix(3, 2, 0.04), helix(6, 2, 0.04), helix(3, 2, 0.01)
    e = [qb.estimate_gib(m, nhist=8) for m in (small, wide, long_)]
    assert 0 < e[0] < e[1] and e[0] < e[2]
    assert qb.estimate_gib(small, nhist=16) > qb.estimate_gib(small, nhist=8)


def test_autotune_modes_are_checked():
    for mode in (-1, 0, 1, 2, 3):
        qb.autotune(mode)
    qb.autotune(1)
    with pytest.raises(ValueError):
        qb.autotune(7)
