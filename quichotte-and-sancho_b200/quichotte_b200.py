"""Python mirror of QUICHOTTE's NEGF entry points on the B200 solver (ctypes over the C ABI).

The reference is a Fortran program whose hot path is called as module procedures
(src/scf.f90, src/self_energies.f90, src/green_functions.f90, common/broyden_mixing.f90,
src/observables.f90). This module exposes the same steps with the same argument meaning:

    Model.load(case_dir)        read_input + build_hamiltonian + setup_leads + setup_hubbard
                                + energy grid   (src/quichotte.f90:224-253)
    Solver(model)               setup_storage + scf_setup_sizes + sigma2_init
    Solver.solve_scf(V, fresh)  solve_scf(Volt, fresh_start, converged)
    Solver.current(V)           Current(Volt, J_up, J_down)
    Solver.observables()        G_less_obs, dosd, trU, trD left by the final sweep
    Solver.initial_vector(V)    sweep(M_INIT2) + pack_gf  (fresh start)
    Solver.residual(V, x)       scf_residual2 / scf_residual1
    Solver.self_energies(x)     sigma2_compute (+ Sigma1)
    invert_batched(A)           invert_complex over a batch
    pack_gf / unpack_gf         common/linear_algebra.f90:155-233
    broyden_solve(...)          common/broyden_mixing.f90:51-184 with a host residual
    run_program(case_dir)       the whole program (bin/quichotte.x drop-in)

Errors follow the reference: a singular Dyson matrix raises SingularMatrixError (the
reference stops with exit code 1); a CUDA or HBM-admission failure raises SolverError.
The CUDA library is required: importing this module on a machine without the built
libqsb200.so raises ImportError, there is no CPU fallback.
"""
import ctypes
import os
import subprocess
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(_HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libqsb200.so")
HOST_PATH = os.path.join(BUILD, "libqs_host.so")
PROGRAM = os.path.join(BUILD, "quichotte_b200")

QS_PREC_FP64, QS_PREC_MIXED = 0, 1

if not os.path.exists(LIB_PATH) or not os.path.exists(HOST_PATH):
    raise ImportError(f"quichotte_b200: built libraries not found in {BUILD}; run "
                      "`python quichotte-and-sancho_b200/build.py` (CUDA 12.9, sm_100a)")

_host = ctypes.CDLL(HOST_PATH, mode=ctypes.RTLD_GLOBAL)
_lib = ctypes.CDLL(LIB_PATH)

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class SolverError(RuntimeError):
    """CUDA failure, HBM admission failure or invalid arguments (status < 0)."""


class SingularMatrixError(SolverError):
    """A Dyson matrix was singular (the reference's ZGETRF INFO > 0, `stop 1`)."""


class _QshModel(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_int) for k in ("N_sites", "Norb", "N_atoms", "order", "n_omega", "n_volt_steps")]
                + [(k, ctypes.c_double) for k in ("V", "Vf", "delv", "T", "mu", "beta", "delta", "w_init", "w_fin",
                                                  "dw", "up", "Ev_min", "Ev_max", "alpha_mix", "tolf", "tolf_order1")]
                + [(k, ctypes.c_int) for k in ("nhist", "maxscf", "continuation", "broyden_single_precision",
                                               "write_hamiltonian", "per_atom")]
                + [(k, _dp) for k in ("H", "GammaL", "GammaR", "U_site", "omega", "Ev")]
                + [("atom_norb", _ip), ("atom_first", _ip), ("model_name", ctypes.c_char * 32),
                   ("input_file", ctypes.c_char * 32)])


class QsProblem(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_int) for k in ("Norb", "N_sites", "N_atoms", "order", "n_omega")]
                + [(k, ctypes.c_void_p) for k in ("H", "GammaL", "GammaR", "U_site", "omega", "atom_norb",
                                                  "atom_first")]
                + [(k, ctypes.c_double) for k in ("mu", "beta", "delta", "alpha_mix", "tolf", "tolf_order1")]
                + [(k, ctypes.c_int) for k in ("nhist", "maxscf", "single_history", "precision", "device")])


class QsScfStep(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int), ("fmax", ctypes.c_double), ("rms", ctypes.c_double), ("nh", ctypes.c_int)]


class QsScfResult(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int), ("n_iter", ctypes.c_int), ("fmax", ctypes.c_double),
                ("aborted", ctypes.c_int), ("runaway", ctypes.c_int), ("unphysical", ctypes.c_int),
                ("i_worst", ctypes.c_int), ("n_worst", ctypes.c_double), ("w_worst", ctypes.c_double),
                ("n_resets", ctypes.c_int), ("log", ctypes.POINTER(QsScfStep)), ("log_cap", ctypes.c_int),
                ("n_log", ctypes.c_int), ("seconds", ctypes.c_double), ("n_mixed", ctypes.c_int)]


RESIDUAL_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int64, _dp, _dp, _ip)

_host.qsh_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(_QshModel)), ctypes.c_char_p, ctypes.c_int,
                           ctypes.c_void_p]
EIGENVALUES_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _ip, ctypes.c_int)
LOWDIN_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int)


class QshSolverApi(ctypes.Structure):
    """qsh_solver_api of qs_host.h (the solver entry points as plain pointers, then the
    optional set-up linear algebra)."""
    _fields_ = ([("name", ctypes.c_char_p)] + [(k, ctypes.c_void_p) for k in ("create", "destroy", "last_error",
                                                                              "solve_scf", "current",
                                                                              "get_observables")]
                + [("hermitian_eigenvalues", EIGENVALUES_FN), ("dftb_lowdin", LOWDIN_FN)])


_host.qsh_load_with.argtypes = [ctypes.c_char_p, ctypes.POINTER(QshSolverApi), ctypes.c_int,
                                ctypes.POINTER(ctypes.POINTER(_QshModel)), ctypes.c_char_p, ctypes.c_int,
                                ctypes.c_void_p]
_host.qsh_helix.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 15 + [ctypes.c_int,
                                                                                     ctypes.POINTER(ctypes.POINTER(_QshModel))]
_host.qsh_free.argtypes = [ctypes.POINTER(_QshModel)]
_host.qsh_fmt_real.argtypes = [ctypes.c_double, ctypes.c_char_p]


def bind_solver(lib, prefix):
    """Declare the qsb200.h signatures on a library whose entry points carry `prefix`."""
    f = lambda name: getattr(lib, prefix + name)
    f("create").argtypes = [ctypes.POINTER(QsProblem), ctypes.POINTER(ctypes.c_void_p)]
    f("destroy").argtypes = [ctypes.c_void_p]
    f("destroy").restype = None
    f("last_error").argtypes = [ctypes.c_void_p]
    f("last_error").restype = ctypes.c_char_p
    f("solve_scf").argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(QsScfResult)]
    f("current").argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp]
    f("get_observables").argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
    f("vector_length").argtypes = [ctypes.c_void_p]
    f("vector_length").restype = ctypes.c_int64
    f("active_states").argtypes = [ctypes.c_void_p]
    f("fft_length").argtypes = [ctypes.c_void_p]
    f("initial_vector").argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    f("residual").argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, _ip]
    f("self_energies").argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p]
    f("invert_batched").argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    f("pack_gf").argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f("unpack_gf").argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f("broyden_solve_host").argtypes = [RESIDUAL_FN, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                        _ip, _ip, _dp, ctypes.POINTER(QsScfStep), ctypes.c_int]
    return lib


bind_solver(_lib, "qs_")
_lib.qs_kernel_launches.restype = ctypes.c_int64
_lib.qs_graph_replays.argtypes = [ctypes.c_void_p]
_lib.qs_graph_replays.restype = ctypes.c_int64
_lib.qs_profile.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
KERNEL_FAMILIES = ("dyson_gj", "keldysh_scf2", "sig2_fwdA", "sig2_mid", "sig2_invC", "final_outputs", "broyden",
                   "reductions", "other")


def kernel_launches():
    """Kernels launched by libqsb200.so in this process so far."""
    return int(_lib.qs_kernel_launches())

# every entry point of include/qsb200.h (the loader test checks they are all exported)
C_ABI = ("qs_create", "qs_destroy", "qs_last_error", "qs_solve_scf", "qs_current", "qs_get_observables",
         "qs_vector_length", "qs_active_states", "qs_fft_length", "qs_initial_vector", "qs_residual",
         "qs_self_energies", "qs_invert_batched", "qs_pack_gf", "qs_unpack_gf", "qs_broyden_solve_host",
         "qs_kernel_launches", "qs_graph_replays", "qs_profile", "qs_invert_batched_noalloc", "qs_estimate_bytes", "qs_device_bytes",
         "qs_server_create", "qs_server_submit", "qs_server_poll", "qs_server_pending", "qs_server_clock",
         "qs_server_budget_gib", "qs_server_destroy", "qs_autotune", "qs_tuned_choice",
         "qs_hermitian_eigensystem", "qs_hermitian_eigenvalues", "qs_dftb_lowdin")
TUNE_DYSON, TUNE_KELDYSH, TUNE_SIG2_A, TUNE_SIG2_C, TUNE_KELDYSH32 = 0, 1, 2, 3, 4
QS_ERR_NOALLOC_LIMIT = -1001
QS_ERR_TOO_LARGE = -1002


class QsServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_inflight", ctypes.c_int), ("hbm_budget_gib", ctypes.c_double)]


class QsRequestResult(ctypes.Structure):
    _fields_ = ([("id", ctypes.c_int64)] + [(k, ctypes.c_int) for k in ("status", "converged", "n_iter", "n_mixed")]
                + [(k, ctypes.c_double) for k in ("fmax", "J_up", "J_down", "solve_s", "t_arrival", "t_start",
                                                  "t_done", "device_gib")] + [("error", ctypes.c_char * 160)])


_lib.qs_autotune.argtypes = [ctypes.c_int]
_lib.qs_tuned_choice.argtypes = [ctypes.c_int, ctypes.c_int]


def autotune(mode):
    """1: time kernel variants per size (default); 0: size heuristics; 2/3: force the first
    (tensor-core/blocked) or last variant; 4: the second of three (the two-blocks-per-SM
    blocked Dyson); -1: forget the recorded choices."""
    if _lib.qs_autotune(mode) != 0:
        raise ValueError(mode)


def tune_key(order, n_omega):
    """The size key of an autotuner decision (matrix order and the octave of the grid)."""
    return order + 1024 * (int(n_omega).bit_length() - 1)


def tuned_choice(kind, size):
    return _lib.qs_tuned_choice(kind, size)


_lib.qs_estimate_bytes.argtypes = [ctypes.POINTER(QsProblem), _dp]
_lib.qs_device_bytes.argtypes = [ctypes.c_void_p]
_lib.qs_device_bytes.restype = ctypes.c_double
_lib.qs_server_create.argtypes = [ctypes.POINTER(QsServerConfig), ctypes.POINTER(ctypes.c_void_p)]
_lib.qs_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(QsProblem), ctypes.c_double, ctypes.c_int64]
_lib.qs_server_poll.argtypes = [ctypes.c_void_p, ctypes.POINTER(QsRequestResult), ctypes.c_int, ctypes.c_double]
_lib.qs_server_pending.argtypes = [ctypes.c_void_p]
_lib.qs_server_clock.argtypes = [ctypes.c_void_p]
_lib.qs_server_clock.restype = ctypes.c_double
_lib.qs_server_budget_gib.argtypes = [ctypes.c_void_p]
_lib.qs_server_budget_gib.restype = ctypes.c_double
_lib.qs_server_destroy.argtypes = [ctypes.c_void_p]
_lib.qs_server_destroy.restype = None
_lib.qs_invert_batched_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]
_lib.qs_hermitian_eigensystem.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_int]
_lib.qs_hermitian_eigenvalues.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_int]
_lib.qs_dftb_lowdin.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                ctypes.c_void_p, _dp, ctypes.c_int]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Model:
    """The model and grid of one input.dat (module globals of Parameters/Hamiltonian/
    GreenFunctions after set-up). Arrays are numpy views copied out of the host layer."""

    def __init__(self, cptr):
        m = cptr.contents
        self._c = cptr
        No, n = m.Norb, m.n_omega
        self.Norb, self.N_sites, self.N_atoms, self.order, self.n_omega = No, m.N_sites, m.N_atoms, m.order, n
        self.n_volt_steps = m.n_volt_steps
        for k in ("V", "Vf", "delv", "T", "mu", "beta", "delta", "w_init", "w_fin", "alpha_mix", "tolf",
                  "tolf_order1"):
            setattr(self, k, getattr(m, k))
        self.nhist, self.maxscf = m.nhist, m.maxscf
        self.continuation, self.single_history = bool(m.continuation), bool(m.broyden_single_precision)
        cp = lambda p, cnt: np.ctypeslib.as_array(p, (cnt,)).copy()
        self.H = cp(m.H, 2 * No * No).view(np.complex128).reshape(No, No, order="F")
        self.GammaL = cp(m.GammaL, 2 * No * No).view(np.complex128).reshape(No, No, order="F")
        self.GammaR = cp(m.GammaR, 2 * No * No).view(np.complex128).reshape(No, No, order="F")
        self.U_site = cp(m.U_site, No)
        self.omega = cp(m.omega, n)
        self.Ev = cp(m.Ev, No)
        self.atom_norb = np.ctypeslib.as_array(m.atom_norb, (m.N_atoms,)).astype(np.int32).copy()
        self.atom_first = np.ctypeslib.as_array(m.atom_first, (m.N_atoms,)).astype(np.int32).copy()
        self.model_name = m.model_name.decode()

    def __del__(self):
        if getattr(self, "_c", None):
            _host.qsh_free(self._c)
            self._c = None

    @classmethod
    def load(cls, case_dir):
        p = ctypes.POINTER(_QshModel)()
        err = ctypes.create_string_buffer(4096)
        rc = _host.qsh_load(os.fsencode(case_dir), ctypes.byref(p), err, 4096, None)
        if rc != 0:
            raise ValueError(err.value.decode(errors="replace").strip())
        return cls(p)

    @classmethod
    def load_with(cls, case_dir, api, device=0):
        """load with the set-up linear algebra of `api` (a QshSolverApi)."""
        p = ctypes.POINTER(_QshModel)()
        err = ctypes.create_string_buffer(4096)
        rc = _host.qsh_load_with(os.fsencode(case_dir), ctypes.byref(api), device, ctypes.byref(p), err, 4096, None)
        if rc != 0:
            raise ValueError(err.value.decode(errors="replace").strip())
        return cls(p)

    @classmethod
    def helix(cls, N_ions, N_turns, hel_length, hel_radius, hand, E_CC, t_hop, lamb, U_int, GammaL_up, GammaL_down,
              GammaR, T, mu, dw, up, delta, order=2):
        p = ctypes.POINTER(_QshModel)()
        rc = _host.qsh_helix(N_ions, N_turns, hel_length, hel_radius, hand, E_CC, t_hop, lamb, U_int, GammaL_up,
                             GammaL_down, GammaR, T, mu, dw, up, delta, order, ctypes.byref(p))
        if rc != 0:
            raise ValueError("invalid helix parameters")
        return cls(p)

    def problem(self, precision=QS_PREC_FP64, device=0, **over):
        """qs_problem for this model (keeps the arrays alive on the returned object)."""
        keep = dict(H=np.asfortranarray(self.H), GammaL=np.asfortranarray(self.GammaL),
                    GammaR=np.asfortranarray(self.GammaR), U=np.ascontiguousarray(self.U_site),
                    omega=np.ascontiguousarray(self.omega), an=self.atom_norb, af=self.atom_first)
        s = dict(alpha_mix=self.alpha_mix, tolf=self.tolf, tolf_order1=self.tolf_order1, nhist=self.nhist,
                 maxscf=self.maxscf, single_history=int(self.single_history))
        s.update(over)
        p = QsProblem(self.Norb, self.N_sites, self.N_atoms, self.order, self.n_omega, _ptr(keep["H"]),
                      _ptr(keep["GammaL"]), _ptr(keep["GammaR"]), _ptr(keep["U"]), _ptr(keep["omega"]),
                      _ptr(keep["an"]), _ptr(keep["af"]), self.mu, self.beta, self.delta, s["alpha_mix"], s["tolf"],
                      s["tolf_order1"], s["nhist"], s["maxscf"], s["single_history"], precision, device)
        p._keep = keep
        return p


class Solver:
    """One solver handle over a library with the qsb200.h entry points (default: the
    B200 library)."""

    def __init__(self, model, precision=QS_PREC_FP64, device=0, lib=None, prefix="qs_", **settings):
        self.lib, self.prefix = (lib or _lib), prefix
        self.model = model
        self._prob = model.problem(precision, device, **settings)
        self._h = ctypes.c_void_p()
        rc = self._f("create")(ctypes.byref(self._prob), ctypes.byref(self._h))
        if rc != 0:
            msg = self._f("last_error")(self._h).decode() if self._h else ""
            if self._h:
                self._f("destroy")(self._h)
                self._h = None
            raise SolverError(f"create failed ({rc}): {msg}")
        self.n_vec = int(self._f("vector_length")(self._h))
        self.nA = int(self._f("active_states")(self._h))
        self.Nf = int(self._f("fft_length")(self._h))

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, rc, what):
        if rc == 0:
            return
        msg = self._f("last_error")(self._h).decode()
        if rc > 0:
            raise SingularMatrixError(f"{what}: {msg}")
        raise SolverError(f"{what} failed ({rc}): {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def graph_replays(self):
        """SCF residuals of this handle replayed from a CUDA graph (qs_graph_replays)."""
        return int(self.lib.qs_graph_replays(self._h)) if self.prefix == "qs_" else 0

    def device_gib(self):
        """Device memory (GiB) this handle has allocated."""
        return self._f("device_bytes")(self._h)

    def solve_scf(self, V, fresh_start=True):
        cap = self.model.maxscf + 2
        log = (QsScfStep * cap)()
        r = QsScfResult()
        r.log, r.log_cap = log, cap
        self._check(self._f("solve_scf")(self._h, V, int(fresh_start), ctypes.byref(r)), "solve_scf")
        out = {k: getattr(r, k) for k in ("converged", "n_iter", "fmax", "aborted", "runaway", "unphysical",
                                           "i_worst", "n_worst", "w_worst", "n_resets", "seconds", "n_mixed")}
        out["converged"] = bool(out["converged"])
        out["log"] = [(log[i].step, log[i].fmax, log[i].rms, log[i].nh) for i in range(r.n_log)]
        return out

    def current(self, V=0.0):
        ju, jd = ctypes.c_double(), ctypes.c_double()
        self._check(self._f("current")(self._h, V, ctypes.byref(ju), ctypes.byref(jd)), "current")
        return ju.value, jd.value

    def observables(self):
        m = self.model
        G = np.zeros((m.Norb, m.Norb), np.complex128, order="F")
        dosd = np.zeros((m.Norb, m.n_omega), np.float64, order="F")
        trU = np.zeros(m.n_omega)
        trD = np.zeros(m.n_omega)
        self._check(self._f("get_observables")(self._h, _ptr(G), _ptr(dosd), _ptr(trU), _ptr(trD)), "observables")
        return dict(G_less_obs=G, dosd=dosd, trU=trU, trD=trD)

    def initial_vector(self, V):
        x = np.zeros(max(self.n_vec, 1))
        self._check(self._f("initial_vector")(self._h, V, _ptr(x)), "initial_vector")
        return x[: self.n_vec]

    def residual(self, V, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        F = np.zeros_like(x)
        ab = ctypes.c_int(0)
        self._check(self._f("residual")(self._h, V, _ptr(x), _ptr(F), ctypes.byref(ab)), "residual")
        return F, bool(ab.value)

    def profile(self, enable):
        """Per-family device time (ms) and launch counts since the last call; enable
        True/False switches event timing on/off, None only reads."""
        ms = np.zeros(len(KERNEL_FAMILIES))
        cnt = np.zeros(len(KERNEL_FAMILIES), np.int64)
        flag = -1 if enable is None else int(bool(enable))
        self._f("profile")(self._h, flag, _ptr(ms), _ptr(cnt), len(KERNEL_FAMILIES))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_FAMILIES)}

    def self_energies(self, x):
        m, nA = self.model, self.nA
        x = np.ascontiguousarray(x, dtype=np.float64)
        SR = np.zeros((nA, nA, m.n_omega), np.complex128, order="F")
        SL = np.zeros_like(SR)
        S1 = np.zeros((m.Norb, m.Norb), np.complex128, order="F")
        self._check(self._f("self_energies")(self._h, _ptr(x), _ptr(SR), _ptr(SL), _ptr(S1)), "self_energies")
        return SR, SL, S1


def estimate_gib(model, precision=QS_PREC_FP64, **settings):
    """Device memory (GiB) a solve of this model keeps (qs_estimate_bytes)."""
    prob = model.problem(precision, 0, **settings)
    g = ctypes.c_double()
    rc = _lib.qs_estimate_bytes(ctypes.byref(prob), ctypes.byref(g))
    if rc != 0:
        raise SolverError(f"estimate failed ({rc})")
    return g.value


class Server:
    """The serving loop (qs_server_*): IV-point requests admitted by HBM budget and solved
    concurrently on the device (continuous batching)."""

    def __init__(self, device=0, max_inflight=4, hbm_budget_gib=0.0):
        cfg = QsServerConfig(device, max_inflight, hbm_budget_gib)
        self._s = ctypes.c_void_p()
        rc = _lib.qs_server_create(ctypes.byref(cfg), ctypes.byref(self._s))
        if rc != 0:
            raise SolverError(f"qs_server_create failed ({rc})")

    @property
    def budget_gib(self):
        return _lib.qs_server_budget_gib(self._s)

    def clock(self):
        return _lib.qs_server_clock(self._s)

    def submit(self, model, V, rid, precision=QS_PREC_FP64, **settings):
        """Queue one IV point; the problem arrays are copied before this returns.
        Returns 0 or QS_ERR_TOO_LARGE (never fits the budget)."""
        prob = model.problem(precision, 0, **settings)
        rc = _lib.qs_server_submit(self._s, ctypes.byref(prob), V, rid)
        if rc not in (0, QS_ERR_TOO_LARGE):
            raise SolverError(f"qs_server_submit failed ({rc})")
        return rc

    def pending(self):
        return _lib.qs_server_pending(self._s)

    def poll(self, timeout=0.0, cap=64):
        buf = (QsRequestResult * cap)()
        k = _lib.qs_server_poll(self._s, buf, cap, timeout)
        out = [{f: getattr(buf[i], f) for f, _ in QsRequestResult._fields_} for i in range(k)]
        for r in out:
            r["error"] = r["error"].decode(errors="replace")
        return out

    def drain(self, timeout=3600.0):
        """Results of every request still pending."""
        out, t0 = [], time.time()
        while self.pending() > 0 and time.time() - t0 < timeout:
            out += self.poll(timeout=1.0)
        return out

    def close(self):
        if getattr(self, "_s", None):
            _lib.qs_server_destroy(self._s)
            self._s = None

    def __del__(self):
        self.close()


def invert_batched(A, precision=QS_PREC_FP64, lib=None, prefix="qs_"):
    """A: (batch, N, N) complex; returns (inverses, info) with info[b] != 0 for a zero pivot."""
    lib = lib or _lib
    A = np.asarray(A, np.complex128)
    batch, N, _ = A.shape
    buf = np.array(A.transpose(0, 2, 1), dtype=np.complex128, order="C", copy=True)  # column-major matrices
    info = np.zeros(batch, np.int32)
    rc = getattr(lib, prefix + "invert_batched")(N, batch, _ptr(buf), _ptr(info), precision)
    if rc < 0:
        raise SolverError(f"invert_batched failed ({rc})")
    return buf.transpose(0, 2, 1).copy(), info


def hermitian_eigensystem(A, device=0):
    """hermitian_eigensystem (zheev) on the device over a batch. A: (batch, N, N) or (N, N)
    Hermitian complex. Returns (E ascending, Z with the eigenvectors in its columns, info)
    with info[b] = 1 for a matrix that did not converge or holds non-finite entries."""
    A = np.asarray(A, np.complex128)
    single = A.ndim == 2
    if single:
        A = A[None]
    batch, N, _ = A.shape
    buf = np.array(A.transpose(0, 2, 1), dtype=np.complex128, order="C", copy=True)
    E = np.zeros((batch, N))
    info = np.zeros(batch, np.int32)
    rc = _lib.qs_hermitian_eigensystem(N, batch, _ptr(buf), _ptr(E), _ptr(info), device)
    if rc < 0:
        raise SolverError(f"hermitian_eigensystem failed ({rc})")
    Z = buf.transpose(0, 2, 1).copy()
    return (E[0], Z[0], info[0]) if single else (E, Z, info)


def hermitian_eigenvalues(A, device=0):
    """Eigenvalues only (zheev JOBZ='N') on the device. A: (batch, N, N) or (N, N) Hermitian
    complex, not modified. Returns (E ascending, info)."""
    A = np.asarray(A, np.complex128)
    single = A.ndim == 2
    if single:
        A = A[None]
    batch, N, _ = A.shape
    buf = np.array(A.transpose(0, 2, 1), dtype=np.complex128, order="C", copy=True)
    E = np.zeros((batch, N))
    info = np.zeros(batch, np.int32)
    rc = _lib.qs_hermitian_eigenvalues(N, batch, _ptr(buf), _ptr(E), _ptr(info), device)
    if rc < 0:
        raise SolverError(f"hermitian_eigenvalues failed ({rc})")
    return (E[0], info[0]) if single else (E, info)


def dftb_lowdin(S, H0, Lam, soc_dual=True, device=0):
    """The Loewdin transform of the dftb_hs model on the device: S, H0 (N, N) real, Lam
    (2N, 2N) complex. Returns (H (2N, 2N) complex, smallest eigenvalue of S); raises for an S
    that is not positive definite, as the reference stops there."""
    S = np.asfortranarray(S, np.float64)
    H0 = np.asfortranarray(H0, np.float64)
    Lam = np.asfortranarray(Lam, np.complex128)
    N = S.shape[0]
    H = np.zeros((2 * N, 2 * N), np.complex128, order="F")
    evmin = ctypes.c_double(0.0)
    rc = _lib.qs_dftb_lowdin(N, _ptr(S), _ptr(H0), _ptr(Lam), int(bool(soc_dual)), _ptr(H), ctypes.byref(evmin),
                             device)
    if rc == 1:
        raise SolverError(f"overlap matrix is not positive definite (min eigenvalue {evmin.value:.3e})")
    if rc != 0:
        raise SolverError(f"dftb_lowdin failed ({rc})")
    return H, evmin.value


def pack_gf(Gr, Gl, lib=None, prefix="qs_"):
    """Gr, Gl: (nb, nb, Nw) complex, Fortran order (the reference's arrays)."""
    lib = lib or _lib
    nb, _, Nw = Gr.shape
    Gr = np.asfortranarray(Gr, np.complex128)
    Gl = np.asfortranarray(Gl, np.complex128)
    out = np.zeros(3 * nb * nb * Nw)
    rc = getattr(lib, prefix + "pack_gf")(nb, Nw, _ptr(Gr), _ptr(Gl), _ptr(out))
    if rc != 0:
        raise SolverError(f"pack_gf failed ({rc})")
    return out


def unpack_gf(x, nb, Nw, lib=None, prefix="qs_"):
    lib = lib or _lib
    x = np.ascontiguousarray(x, np.float64)
    Gr = np.zeros((nb, nb, Nw), np.complex128, order="F")
    Gl = np.zeros_like(Gr)
    rc = getattr(lib, prefix + "unpack_gf")(nb, Nw, _ptr(x), _ptr(Gr), _ptr(Gl))
    if rc != 0:
        raise SolverError(f"unpack_gf failed ({rc})")
    return Gr, Gl


def broyden_solve(residual, x0, alpha_mix=0.5, nhist=16, maxscf=300, tolf=1e-6, single_history=True, lib=None,
                  prefix="qs_"):
    """broyden_solve with residual(x) -> (F, abort) evaluated in Python on host arrays."""
    lib = lib or _lib
    x = np.ascontiguousarray(x0, np.float64).copy()
    n = x.size

    def cb(ctx, nn, xp, Fp, abp):
        xv = np.ctypeslib.as_array(xp, (nn,))
        F, ab = residual(xv.copy())
        np.ctypeslib.as_array(Fp, (nn,))[:] = F
        abp[0] = int(bool(ab))

    fn = RESIDUAL_FN(cb)
    conv, nit, fmax = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    log = (QsScfStep * (maxscf + 1))()
    rc = getattr(lib, prefix + "broyden_solve_host")(fn, None, _ptr(x), n, alpha_mix, nhist, maxscf, tolf,
                                                      int(single_history), ctypes.byref(conv), ctypes.byref(nit),
                                                      ctypes.byref(fmax), log, maxscf + 1)
    if rc != 0:
        raise SolverError(f"broyden_solve failed ({rc})")
    steps = [(log[i].step, log[i].fmax, log[i].rms, log[i].nh) for i in range(nit.value)]
    return x, bool(conv.value), nit.value, fmax.value, steps


def run_program(case_dir, device=0, timeout=3600):
    """Run the QUICHOTTE program (quichotte_b200) in case_dir; returns its exit code."""
    env = dict(os.environ, QS_DEVICE=str(device))
    with open(os.path.join(case_dir, "stdout.txt"), "w") as out:
        return subprocess.run([PROGRAM, case_dir], stdout=out, stderr=subprocess.STDOUT, env=env,
                              timeout=timeout).returncode
