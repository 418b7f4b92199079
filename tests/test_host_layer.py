"""The host layer (input.dat, models, grid, output format) against the reference's
golden files (CPU only)."""
import ctypes
import math
import os
import random

import numpy as np
import pytest

import golden_runner as g
import quichotte_b200 as qb

CASES = os.path.join(g.GOLDEN, "cases")


def test_list_directed_format_reproduces_golden_lines():
    import ctypes
    buf = ctypes.create_string_buffer(64)

    def fmt(x):
        qb._host.qsh_fmt_real(x, buf)
        return buf.value.decode()

    for case in ("order2_second_order", "order2_dftb_hs", "order0_dftb_blocks"):
        for name in os.listdir(os.path.join(CASES, case, "reference")):
            if name == "hamiltonian_matrix.dat":
                continue
            for line in open(os.path.join(CASES, case, "reference", name)):
                line = line.rstrip("\n")
                toks = line.split()
                out = ""
                for i, t in enumerate(toks):
                    if "." in t or "E" in t:
                        out += fmt(float(t))
                    else:
                        out += f" {int(t):11d}"
                assert out == line


@pytest.mark.parametrize("case", ["error_N_sites_mismatch", "error_unknown_hamiltonian", "error_dftb_lead_overlap",
                                  "error_dftb_hs_no_lmax"])
def test_bad_inputs_are_rejected(case):
    with pytest.raises(ValueError):
        qb.Model.load(os.path.join(CASES, case))


def test_legacy_input_name_and_aliases():
    m = qb.Model.load(os.path.join(CASES, "legacy_inputSOC"))
    assert m.order == 1 and m.alpha_mix == 0.5 and m.Norb == 8
    assert np.all(m.U_site[::2] == 0.8)


def test_dftb_hs_hamiltonian_matches_golden():
    m = qb.Model.load(os.path.join(CASES, "order2_dftb_hs"))
    ref = np.loadtxt(os.path.join(CASES, "order2_dftb_hs", "reference", "hamiltonian_matrix.dat"))
    H = np.zeros_like(m.H)
    for i, j, re, im in ref:
        H[int(i) - 1, int(j) - 1] = re + 1j * im
    assert np.max(np.abs(H - m.H)) < 1e-12
    assert np.allclose(m.H, m.H.conj().T, atol=0)


def test_helix_grid_and_hermiticity():
    m = qb.Model.load(os.path.join(CASES, "order2_second_order"))
    ev = np.linalg.eigvalsh(m.H)
    w_init = ev[0] - 1.0
    n = int((ev[-1] + 1.0 - w_init) / m.delta)
    assert m.n_omega == n == 329
    assert np.allclose(m.omega, w_init + m.delta * np.arange(1, n + 1), atol=1e-12)
    assert np.allclose(m.H, m.H.conj().T, atol=0)
    # leads on site 1 (spin-dependent) and the last site
    assert m.GammaL[0, 0] == 1.5 and m.GammaL[1, 1] == 1.0 and m.GammaR[-1, -1] == 1.0


def test_site_dependent_U():
    m = qb.Model.load(os.path.join(CASES, "order2_lefthanded_siteU"))
    assert list(m.U_site[::2]) == [0.8, 0.6, 0.6, 0.8] and not m.U_site[1::2].any()


def _printf_rules(x):
    """gfortran list-directed REAL(8) layout, written with printf-style formatting."""
    if x == 0.0:
        v = "%.16f" % 0.0
        if math.copysign(1.0, x) < 0:
            v = "-" + v
        return " %20s     " % v
    m = "%.16E" % x
    e = int(m.split("E")[1])
    if -1 <= e < 17:
        return " %20s     " % ("%.*f" % (16 - e, x))
    return " %25s" % (m.split("E")[0] + "E%s%03d" % ("-" if e < 0 else "+", abs(e)))


def test_fast_formatter_matches_the_printf_rules():
    """qsh_fmt_real (std::to_chars digits) against the same rules written with printf, on
    random magnitudes and the F/E boundaries, signed zeros and extremes."""
    rnd = random.Random(3)
    vals = [rnd.uniform(-1, 1) * 10 ** rnd.uniform(-40, 40) for _ in range(20000)]
    vals += [0.1, -0.1, 0.09999999999999999, 1e17, -1e17, 9.999999999999998e16, 1.0, 0.0, -0.0, 1e-300, 5e-324,
             1.7976931348623157e308, 2.5e-7, 123456.789]
    lib = ctypes.CDLL(qb.HOST_PATH)
    lib.qsh_fmt_real.argtypes = [ctypes.c_double, ctypes.c_char_p]
    buf = ctypes.create_string_buffer(64)
    for x in vals:
        lib.qsh_fmt_real(x, buf)
        assert buf.value.decode() == _printf_rules(x), repr(x)


def _numpy_setup_api(calls, fail_eigensystem=False):
    """A qsh_solver_api whose set-up linear algebra is LAPACK through numpy (the solver
    entry points stay NULL: only the model set-up runs)."""
    def eigenvalues(N, batch, A, E, info, device):
        calls.append("eigenvalues")
        if fail_eigensystem:
            info[0] = 1
            return 1
        a = np.ctypeslib.as_array(A, (batch * N * N * 2,)).view(np.complex128).reshape(batch, N, N)
        e = np.ctypeslib.as_array(E, (batch * N,)).reshape(batch, N)
        for b in range(batch):
            e[b] = np.linalg.eigvalsh(a[b].T)  # column-major storage
            info[b] = 0
        return 0

    def lowdin(N, S, H0, Lam, dual, H, evmin, device):
        calls.append("lowdin")
        s = np.ctypeslib.as_array(S, (N * N,)).reshape(N, N).T
        h0 = np.ctypeslib.as_array(H0, (N * N,)).reshape(N, N).T
        lam = np.ctypeslib.as_array(Lam, (8 * N * N,)).view(np.complex128).reshape(2 * N, 2 * N).T
        ev, U = np.linalg.eigh(s)
        evmin[0] = ev.min()
        W = U / np.sqrt(np.sqrt(ev))
        Sx2, Sm2 = np.kron(s, np.eye(2)), np.kron(W @ W.T, np.eye(2))
        Hao = np.kron(h0, np.eye(2)) + (0.5 * (Sx2 @ lam + lam @ Sx2) if dual else lam)
        Hn = Sm2 @ Hao @ Sm2
        out = np.ctypeslib.as_array(H, (8 * N * N,)).view(np.complex128).reshape(2 * N, 2 * N)
        out[:] = (0.5 * (Hn + Hn.conj().T)).T
        return 0
    api = qb.QshSolverApi()
    api.name = b"numpy-setup"
    api.hermitian_eigenvalues = qb.EIGENVALUES_FN(eigenvalues)
    api.dftb_lowdin = qb.LOWDIN_FN(lowdin)
    api._keep = (api.hermitian_eigenvalues, api.dftb_lowdin)
    return api


@pytest.mark.parametrize("case", ["order2_dftb_hs", "order2_second_order"])
def test_model_setup_through_the_solver_api(case):
    """qsh_load_with hands the grid eigenproblem and the dftb_hs Loewdin transform to the
    solver's set-up entry points (the B200 program passes qs_hermitian_eigenvalues and
    qs_dftb_lowdin); with LAPACK behind them the model equals the host-built one."""
    calls = []
    api = _numpy_setup_api(calls)
    m = qb.Model.load_with(os.path.join(CASES, case), api)
    h = qb.Model.load(os.path.join(CASES, case))
    assert calls == (["lowdin", "eigenvalues"] if case == "order2_dftb_hs" else ["eigenvalues"])
    assert np.max(np.abs(m.H - h.H)) <= 1e-12 * np.max(np.abs(h.H))
    assert np.max(np.abs(m.Ev - h.Ev)) <= 1e-12 * np.max(np.abs(h.Ev))
    assert m.n_omega == h.n_omega
    assert np.max(np.abs(m.omega - h.omega)) <= 1e-12 * np.max(np.abs(h.omega))  # w_init = Ev_min - dw


def test_model_setup_failure_is_the_reference_stop():
    api = _numpy_setup_api([], fail_eigensystem=True)
    with pytest.raises(ValueError, match="ZHEEV eigenproblem failed"):
        qb.Model.load_with(os.path.join(CASES, "order2_second_order"), api)
