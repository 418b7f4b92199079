"""The drop-in boundary: the C-ABI library loads and exports every entry point that
include/qsb200.h and include/qsa200.h declare (no GPU work here)."""
import ctypes
import os
import re

import pytest

import quichotte_b200 as qb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qs[ha]?h?_[a-z0-9_]+)\s*\(", text)))


def test_cuda_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(qb.LIB_PATH)
    names = declared("qsb200.h")
    assert len(names) >= 16
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(qb.C_ABI) <= set(names)


def test_cuda_library_exports_every_sancho_entry_point():
    import sancho_b200 as sb
    lib = ctypes.CDLL(qb.LIB_PATH)
    names = [n for n in declared("qsa200.h") if n.startswith("qsa_")]
    assert len(names) == 11
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(sb.C_ABI) == set(names)


def test_host_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(qb.HOST_PATH)
    names = [n for n in declared("qs_host.h") if n.startswith("qsh_")]
    names += [n for n in declared("qsa_host.h") if n.startswith("qsah_")]
    assert any(n.startswith("qsah_") for n in names)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_program_binaries_are_built():
    import sancho_b200 as sb
    assert os.access(qb.PROGRAM, os.X_OK)
    assert os.access(sb.PROGRAM, os.X_OK)


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
    for mode in (-1, 0, 1, 2, 3, 4):
        qb.autotune(mode)
    qb.autotune(1)
    with pytest.raises(ValueError):
        qb.autotune(7)


C_CLIENT = r"""
/* A plain C99 client of the two headers: every declared entry point is taken by address
 * (so each prototype is valid C and resolves at link time), then the calls that need no
 * GPU run: the memory estimate of a small problem and the list-directed formatter. */
#include <stdio.h>
#include <string.h>
#include "qsb200.h"
#include "qs_host.h"
#include "qsa200.h"
#include "qsa_host.h"

int main(void) {
    void *table[] = {
%TABLE%
    };
    size_t k, n = sizeof table / sizeof table[0];
    for (k = 0; k < n; k++)
        if (!table[k]) return 10;
    {
        enum { NO = 4 };
        double H[2 * NO * NO], GL[2 * NO * NO], GR[2 * NO * NO], U[NO] = {1, 0, 1, 0}, w[64];
        int an[2] = {2, 2}, af[2] = {1, 2};
        qs_problem p;
        double gib = -1.0;
        memset(H, 0, sizeof H); memset(GL, 0, sizeof GL); memset(GR, 0, sizeof GR);
        for (k = 0; k < 64; k++) w[k] = -3.0 + 0.1 * (double)k;
        memset(&p, 0, sizeof p);
        p.Norb = NO; p.N_sites = 2; p.N_atoms = 2; p.order = 2; p.n_omega = 64;
        p.H = H; p.GammaL = GL; p.GammaR = GR; p.U_site = U; p.omega = w;
        p.atom_norb = an; p.atom_first = af;
        p.mu = 0.0; p.beta = 38.7; p.delta = 0.1; p.alpha_mix = 0.1; p.tolf = 1e-8; p.tolf_order1 = 1e-8;
        p.nhist = 4; p.maxscf = 10; p.single_history = 1; p.precision = QS_PREC_FP64; p.device = 0;
        if (qs_estimate_bytes(&p, &gib) != 0 || !(gib > 0.0)) return 11;
    }
    {
        char buf[64];
        qsh_fmt_real(0.5, buf);
        printf("%s|\n", buf);
    }
    return 0;
}
"""


def test_headers_are_plain_c_and_link(tmp_path):
    """The boundary is a C ABI: a C99 program that includes both headers, references every
    declared entry point and links against the two libraries builds with -Wall -Werror and
    runs the calls that need no GPU."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    names = declared("qsb200.h") + [n for n in declared("qs_host.h") if n.startswith("qsh_")]
    names += declared("qsa200.h") + [n for n in declared("qsa_host.h") if n.startswith("qsah_")]
    src = tmp_path / "client.c"
    src.write_text(C_CLIENT.replace("%TABLE%", ",\n".join(f"        (void *)&{n}" for n in names)))
    exe = tmp_path / "client"
    libdir = os.path.dirname(qb.LIB_PATH)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                        str(src), "-o", str(exe), "-L" + libdir, "-lqsb200", "-lqs_host", "-Wl,-rpath," + libdir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, (run.returncode, run.stderr)
    assert run.stdout.strip().endswith("|") and "0.5" in run.stdout
