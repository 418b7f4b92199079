"""Python access to the CPU oracle without the product (TEST AND BASELINE INFRASTRUCTURE).

The CPU oracle (oracle.cpp, built by oracle/build.py into oracle/_build/liboracle.so) is the
checker of the B200 solver and the CPU baseline of the benchmark. This module drives it
through ctypes with the model arrays built here in numpy, so that the timed CPU baseline
loads nothing but liboracle.so and the OpenBLAS it links (never the B200 library or the
host layer).

The model is the reference's analytic helix (paths relative to the reference project):
  helix_coordinate / soc_matrix_elements / build_helix_hamiltonian  src/hamiltonian.f90:83-163
  setup_leads (default contacts: the first and the last site)        src/input_output.f90:310-346
  setup_hubbard (uniform U on the spin-up index of every site)       src/input_output.f90:432-462
  beta = 1/(kB T), Norb = 2 N_sites                                  src/input_output.f90:123-124
  energy grid omega_i = w_init + i delta, i = 1..n_omega             src/quichotte.f90:81-93
with kB from common/constants.f90:19. The grid is given here directly by its first point
w_init and spacing delta (the reference derives w_init from the spectrum of H and dw).
"""
import ctypes
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
KB = 8.6173303e-5  # eV/K (common/constants.f90:19)


def helix_hamiltonian(N_ions, N_turns, hel_length, hel_radius, hand, E_CC, t_hop, lamb):
    """build_helix_hamiltonian (src/hamiltonian.f90:126-163): Norb x Norb complex H, spin
    fastest (state 2i-1 = site i spin up, 2i = spin down, 1-based)."""
    Nat = N_ions * N_turns
    Norb = 2 * Nat
    H = np.zeros((Norb, Norb), np.complex128)

    def coord(i):  # helix_coordinate, 1-based site index
        ang = hand * (i - 1) * 2 * np.pi / N_ions
        return np.array([hel_radius * np.cos(ang), hel_radius * np.sin(ang),
                         hel_length * (i - 1) / (N_turns * (N_ions - 1))])

    for i in range(1, Nat + 1):
        ii = 2 * i  # 1-based spin-down state of site i
        H[ii - 2, ii - 2] = E_CC
        H[ii - 1, ii - 1] = E_CC
        if i <= Nat - 1:
            jj = 2 * (i + 1)
            H[ii - 2, jj - 2] = t_hop
            H[ii - 1, jj - 1] = t_hop
        if i <= Nat - 2:
            jj = 2 * (i + 2)
            r, r1, r2 = coord(i), coord(i + 1), coord(i + 2)
            d1 = (r - r1) / np.linalg.norm(r - r1)
            d2 = (r - r2) / np.linalg.norm(r - r2)
            v = np.cross(d1, d2)
            H[ii - 2, jj - 2] = 1j * lamb * v[2]
            H[ii - 2, jj - 1] = 1j * lamb * (v[0] - 1j * v[1])
            H[ii - 1, jj - 2] = 1j * lamb * (v[0] + 1j * v[1])
            H[ii - 1, jj - 1] = 1j * lamb * (-v[2])
    # make_hermitian: the lower triangle from the upper one
    iu = np.triu_indices(Norb)
    L = np.zeros_like(H)
    L[iu] = H[iu]
    H = L + np.conj(np.triu(L, 1)).T
    return H


class Helix:
    """The analytic helix model with wide-band leads on the first and last site, uniform U,
    and an explicit energy grid (the arrays the reference's module globals hold)."""

    def __init__(self, N_ions, N_turns, hel_length, hel_radius, hand, E_CC, t_hop, lamb, U_int, GammaL_up,
                 GammaL_down, GammaR, T, mu, w_init, delta, n_omega, order=2):
        self.N_sites = N_ions * N_turns
        self.Norb = 2 * self.N_sites
        self.N_atoms = self.N_sites
        self.order = order
        self.H = helix_hamiltonian(N_ions, N_turns, hel_length, hel_radius, hand, E_CC, t_hop, lamb)
        No = self.Norb
        self.GammaL = np.zeros((No, No), np.complex128)
        self.GammaR = np.zeros((No, No), np.complex128)
        self.GammaL[0, 0], self.GammaL[1, 1] = GammaL_up, GammaL_down
        self.GammaR[No - 2, No - 2] = self.GammaR[No - 1, No - 1] = GammaR
        self.U_site = np.zeros(No)
        self.U_site[0::2] = U_int
        self.mu, self.beta, self.delta = mu, 1.0 / (KB * T), delta
        self.n_omega = n_omega
        self.omega = w_init + delta * np.arange(1, n_omega + 1)
        self.atom_norb = np.ones(self.N_atoms, np.int32)
        self.atom_first = np.arange(1, self.N_atoms + 1, dtype=np.int32)


class _Problem(ctypes.Structure):
    """qs_problem of include/qsb200.h."""
    _fields_ = ([(k, ctypes.c_int) for k in ("Norb", "N_sites", "N_atoms", "order", "n_omega")]
                + [(k, ctypes.c_void_p) for k in ("H", "GammaL", "GammaR", "U_site", "omega", "atom_norb",
                                                  "atom_first")]
                + [(k, ctypes.c_double) for k in ("mu", "beta", "delta", "alpha_mix", "tolf", "tolf_order1")]
                + [(k, ctypes.c_int) for k in ("nhist", "maxscf", "single_history", "precision", "device")])


class _Step(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int), ("fmax", ctypes.c_double), ("rms", ctypes.c_double), ("nh", ctypes.c_int)]


class _Result(ctypes.Structure):
    """qs_scf_result of include/qsb200.h."""
    _fields_ = [("converged", ctypes.c_int), ("n_iter", ctypes.c_int), ("fmax", ctypes.c_double),
                ("aborted", ctypes.c_int), ("runaway", ctypes.c_int), ("unphysical", ctypes.c_int),
                ("i_worst", ctypes.c_int), ("n_worst", ctypes.c_double), ("w_worst", ctypes.c_double),
                ("n_resets", ctypes.c_int), ("log", ctypes.POINTER(_Step)), ("log_cap", ctypes.c_int),
                ("n_log", ctypes.c_int), ("seconds", ctypes.c_double), ("n_mixed", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(f"oracle library not built: {LIB} (python oracle/build.py)")
        L = ctypes.CDLL(LIB)
        L.qso_create.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(ctypes.c_void_p)]
        L.qso_destroy.argtypes = [ctypes.c_void_p]
        L.qso_destroy.restype = None
        L.qso_last_error.argtypes = [ctypes.c_void_p]
        L.qso_last_error.restype = ctypes.c_char_p
        L.qso_solve_scf.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_Result)]
        L.qso_current.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
        L.qso_residual.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.POINTER(ctypes.c_int)]
        L.qso_initial_vector.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        L.qso_vector_length.argtypes = [ctypes.c_void_p]
        L.qso_vector_length.restype = ctypes.c_int64
        L.qso_solve_scf_timed.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_Result),
                                          ctypes.c_void_p, ctypes.c_int]
        L.qso_broyden_seconds_per_step.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        L.qso_broyden_seconds_per_step.restype = ctypes.c_double
        _lib = L
    return _lib


class Solver:
    """One oracle solver (qso_create ... qso_destroy) for a model with the arrays above."""

    def __init__(self, model, alpha_mix=0.5, nhist=16, tolf=1e-6, maxscf=300, single_history=1, tolf_order1=1e-8):
        L = lib()
        m = model
        self._keep = [np.asfortranarray(m.H), np.asfortranarray(m.GammaL), np.asfortranarray(m.GammaR),
                      np.ascontiguousarray(m.U_site, np.float64), np.ascontiguousarray(m.omega, np.float64),
                      np.ascontiguousarray(m.atom_norb, np.int32), np.ascontiguousarray(m.atom_first, np.int32)]
        ptr = [a.ctypes.data_as(ctypes.c_void_p) for a in self._keep]
        self._p = _Problem(m.Norb, m.N_sites, m.N_atoms, m.order, m.n_omega, *ptr, m.mu, m.beta, m.delta,
                           alpha_mix, tolf, tolf_order1, nhist, maxscf, int(single_history), 0, 0)
        self.maxscf = maxscf
        self._h = ctypes.c_void_p()
        rc = L.qso_create(ctypes.byref(self._p), ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"qso_create failed ({rc})")
        self.n_vec = int(L.qso_vector_length(self._h))

    def solve_scf(self, V, fresh_start=True):
        L = lib()
        cap = self.maxscf + 2
        log = (_Step * cap)()
        r = _Result()
        r.log, r.log_cap = log, cap
        t = time.perf_counter()
        rc = L.qso_solve_scf(self._h, V, int(fresh_start), ctypes.byref(r))
        wall = time.perf_counter() - t
        if rc != 0:
            raise RuntimeError(f"qso_solve_scf failed ({rc}): {L.qso_last_error(self._h).decode()}")
        return {"converged": bool(r.converged), "n_iter": r.n_iter, "fmax": r.fmax, "aborted": r.aborted,
                "unphysical": r.unphysical, "n_resets": r.n_resets, "wall": wall,
                "log": [(log[i].step, log[i].fmax, log[i].rms, log[i].nh) for i in range(r.n_log)]}

    def solve_timed(self, V, fresh_start=True):
        """solve_scf with the wall time of every SCF iteration (residual + Broyden update):
        returns (result as solve_scf, seconds per iteration; the final sweep excluded)."""
        L = lib()
        cap = self.maxscf + 2
        log = (_Step * cap)()
        r = _Result()
        r.log, r.log_cap = log, cap
        dt = np.zeros(cap)
        k = L.qso_solve_scf_timed(self._h, V, int(fresh_start), ctypes.byref(r), dt.ctypes.data_as(ctypes.c_void_p),
                                  cap)
        if k < 0:
            raise RuntimeError(f"qso_solve_scf_timed failed ({k})")
        res = {"converged": bool(r.converged), "n_iter": r.n_iter, "aborted": r.aborted,
               "log": [(log[i].step, log[i].fmax, log[i].rms, log[i].nh) for i in range(r.n_log)]}
        return res, dt[:k].copy()

    def current(self, V):
        ju, jd = ctypes.c_double(), ctypes.c_double()
        lib().qso_current(self._h, V, ctypes.byref(ju), ctypes.byref(jd))
        return ju.value, jd.value

    def residual(self, V, x):
        x = np.ascontiguousarray(x, np.float64)
        F = np.zeros_like(x)
        ab = ctypes.c_int(0)
        lib().qso_residual(self._h, V, x.ctypes.data_as(ctypes.c_void_p), F.ctypes.data_as(ctypes.c_void_p),
                           ctypes.byref(ab))
        return F, bool(ab.value)

    def initial_vector(self, V):
        x = np.zeros(max(self.n_vec, 1))
        lib().qso_initial_vector(self._h, V, x.ctypes.data_as(ctypes.c_void_p))
        return x[: self.n_vec]

    def close(self):
        if getattr(self, "_h", None):
            lib().qso_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ---- SANCHO (the spinless chain; paths relative to the reference project's SANCHO/) ----

class SanchoChain:
    """The chain model of SANCHO's input (SANCHO/src/hamiltonian.f90:35-137: E_CC on the
    diagonal, t_hop between neighbours; leads GammaL on site 1 and GammaR on the last site;
    uniform U, SANCHO/src/input_output.f90:106-132) and its grid (SANCHO/src/sancho.f90:
    58-92: w_init = min eig(H) - dw, n = int((max eig(H) + up - w_init)/delta),
    omega_i = w_init + i delta)."""

    def __init__(self, N_sites, E_CC, t_hop, U_int, GammaL, GammaR, T, mu, dw, up, delta, order):
        n = N_sites
        H = np.zeros((n, n), np.complex128)
        for i in range(n):
            H[i, i] = E_CC
            if i + 1 < n:
                H[i, i + 1] = H[i + 1, i] = t_hop
        self.N_sites, self.order, self.H = n, order, np.asfortranarray(H)
        self.GammaL = np.zeros((n, n), np.complex128, order="F")
        self.GammaR = np.zeros((n, n), np.complex128, order="F")
        self.GammaL[0, 0] = GammaL
        self.GammaR[n - 1, n - 1] = GammaR
        self.U_site = np.full(n, float(U_int))
        ev = np.linalg.eigvalsh(H)
        w_init, w_fin = ev[0] - dw, ev[-1] + up
        self.n_omega = int((w_fin - w_init) / delta)
        self.omega = w_init + delta * np.arange(1, self.n_omega + 1)
        self.mu, self.beta, self.delta = mu, 1.0 / (KB * T), delta


class _SanchoProblem(ctypes.Structure):
    """qsa_problem of include/qsa200.h."""
    _fields_ = ([(k, ctypes.c_int) for k in ("N_sites", "order", "n_omega")]
                + [(k, ctypes.c_void_p) for k in ("H", "GammaL", "GammaR", "U_site", "omega")]
                + [(k, ctypes.c_double) for k in ("mu", "beta", "delta", "alpha_mix", "tolf")]
                + [(k, ctypes.c_int) for k in ("nhist", "maxscf", "device")])


class SanchoSolver:
    """One SANCHO oracle solver (qsao_create ... qsao_destroy)."""

    def __init__(self, model, alpha_mix=0.3, nhist=8, tolf=1e-6, maxscf=200):
        L = lib()
        for name, args, res in (("qsao_create", [ctypes.POINTER(_SanchoProblem), ctypes.POINTER(ctypes.c_void_p)], None),
                                ("qsao_destroy", [ctypes.c_void_p], "void"),
                                ("qsao_vector_length", [ctypes.c_void_p], ctypes.c_int64),
                                ("qsao_solve_scf", [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                                    ctypes.POINTER(_Result)], None),
                                ("qsao_residual", [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.POINTER(ctypes.c_int)], None),
                                ("qsao_initial_vector", [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p], None)):
            f = getattr(L, name)
            f.argtypes = args
            if res == "void":
                f.restype = None
            elif res is not None:
                f.restype = res
        m = model
        self._keep = [np.asfortranarray(m.H), np.asfortranarray(m.GammaL), np.asfortranarray(m.GammaR),
                      np.ascontiguousarray(m.U_site, np.float64), np.ascontiguousarray(m.omega, np.float64)]
        ptr = [a.ctypes.data_as(ctypes.c_void_p) for a in self._keep]
        self._p = _SanchoProblem(m.N_sites, m.order, m.n_omega, *ptr, m.mu, m.beta, m.delta, alpha_mix, tolf, nhist,
                                 maxscf, 0)
        self.maxscf = maxscf
        self._h = ctypes.c_void_p()
        if L.qsao_create(ctypes.byref(self._p), ctypes.byref(self._h)) != 0:
            raise RuntimeError("qsao_create failed")
        self.n_vec = int(L.qsao_vector_length(self._h))

    def solve_scf(self, V, fresh_start=True):
        cap = self.maxscf + 2
        log = (_Step * cap)()
        r = _Result()
        r.log, r.log_cap = log, cap
        t = time.perf_counter()
        rc = lib().qsao_solve_scf(self._h, V, int(fresh_start), ctypes.byref(r))
        if rc != 0:
            raise RuntimeError(f"qsao_solve_scf failed ({rc})")
        return {"converged": bool(r.converged), "n_iter": r.n_iter, "wall": time.perf_counter() - t}

    def initial_vector(self, V):
        x = np.zeros(self.n_vec)
        lib().qsao_initial_vector(self._h, V, x.ctypes.data_as(ctypes.c_void_p))
        return x

    def residual(self, V, x):
        x = np.ascontiguousarray(x, np.float64)
        F = np.zeros_like(x)
        ab = ctypes.c_int(0)
        lib().qsao_residual(self._h, V, x.ctypes.data_as(ctypes.c_void_p), F.ctypes.data_as(ctypes.c_void_p),
                            ctypes.byref(ab))
        return F, bool(ab.value)

    def close(self):
        if getattr(self, "_h", None):
            lib().qsao_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
