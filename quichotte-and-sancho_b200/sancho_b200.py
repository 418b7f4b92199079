"""Python mirror of SANCHO's entry points on the B200 solver (ctypes over include/qsa200.h).

SANCHO (the reference project's SANCHO/ directory) is a spinless chain solved to third
order in U. Its hot path is called as module procedures (src/scf.f90,
src/self_energies.f90, src/green_functions.f90, src/observables.f90); this module exposes
the same steps with the same argument meaning:

    SanchoModel.load(case_dir)        read_input + build_hamiltonian + leads + setup_hubbard
                                      + energy grid   (src/sancho.f90:58-92)
    SanchoSolver(model)               storage of G_in, G_out and the SCF vector
    SanchoSolver.solve_scf(V, fresh)  solve_scf(Volt, fresh_start, converged)
    SanchoSolver.current(V)           Current(Volt)
    SanchoSolver.observables()        G^<_ii(t=0) and the spectral function
    SanchoSolver.initial_vector(V)    noninteracting_gr_ga + noninteracting_gl_gg + pack_gf
    SanchoSolver.residual(V, x)       scf_residual
    SanchoSolver.self_energies(x)     build_self_energies (Sigma2, Sigma3)
    run_program(case_dir)             the whole program (bin/sancho.x drop-in)

Errors as in quichotte_b200: SingularMatrixError for a singular Dyson matrix, SolverError
for CUDA or argument failures. The CUDA library is required (no CPU fallback).
"""
import ctypes
import os
import subprocess

import numpy as np

import quichotte_b200 as qb

PROGRAM = os.path.join(qb.BUILD, "sancho_b200")
_dp = ctypes.POINTER(ctypes.c_double)
_ptr = qb._ptr

# every entry point of include/qsa200.h
C_ABI = ("qsa_create", "qsa_destroy", "qsa_last_error", "qsa_vector_length", "qsa_solve_scf", "qsa_current",
         "qsa_get_observables", "qsa_initial_vector", "qsa_residual", "qsa_self_energies", "qsa_profile")
KERNEL_FAMILIES = ("dyson", "keldysh", "bubbles", "products", "sigma", "unused", "broyden", "reductions", "other")


class _QsahModel(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_int) for k in ("N_sites", "order", "n_omega", "n_volt_steps", "nhist", "maxscf",
                                             "continuation")]
                + [(k, ctypes.c_double) for k in ("V", "Vf", "delv", "T", "mu", "beta", "delta", "w_init", "w_fin",
                                                  "dw", "up", "alpha_mix", "tolf")]
                + [(k, _dp) for k in ("H", "GammaL", "GammaR", "U_site", "omega", "Ev")]
                + [("model_name", ctypes.c_char * 32)])


class QsaProblem(ctypes.Structure):
    _fields_ = ([(k, ctypes.c_int) for k in ("N_sites", "order", "n_omega")]
                + [(k, ctypes.c_void_p) for k in ("H", "GammaL", "GammaR", "U_site", "omega")]
                + [(k, ctypes.c_double) for k in ("mu", "beta", "delta", "alpha_mix", "tolf")]
                + [(k, ctypes.c_int) for k in ("nhist", "maxscf", "device")])


_host = qb._host
_host.qsah_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(_QsahModel)), ctypes.c_char_p,
                            ctypes.c_int, ctypes.c_void_p]
_host.qsah_free.argtypes = [ctypes.POINTER(_QsahModel)]


def bind_solver(lib, prefix):
    """Declare the qsa200.h signatures on a library whose entry points carry `prefix`."""
    f = lambda name: getattr(lib, prefix + name)
    f("create").argtypes = [ctypes.POINTER(QsaProblem), ctypes.POINTER(ctypes.c_void_p)]
    f("destroy").argtypes = [ctypes.c_void_p]
    f("destroy").restype = None
    f("last_error").argtypes = [ctypes.c_void_p]
    f("last_error").restype = ctypes.c_char_p
    f("vector_length").argtypes = [ctypes.c_void_p]
    f("vector_length").restype = ctypes.c_int64
    f("solve_scf").argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(qb.QsScfResult)]
    f("current").argtypes = [ctypes.c_void_p, ctypes.c_double, _dp]
    f("get_observables").argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f("initial_vector").argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    f("residual").argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.POINTER(ctypes.c_int)]
    f("self_energies").argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
    if hasattr(lib, prefix + "profile"):
        f("profile").argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    return lib


bind_solver(qb._lib, "qsa_")


class SanchoModel:
    """The chain and grid of one SANCHO input.dat (arrays copied out of the host layer)."""

    def __init__(self, cptr):
        m = cptr.contents
        self._c = cptr
        Na, n = m.N_sites, m.n_omega
        self.N_sites, self.order, self.n_omega, self.n_volt_steps = Na, m.order, n, m.n_volt_steps
        for k in ("V", "Vf", "delv", "T", "mu", "beta", "delta", "w_init", "w_fin", "dw", "up", "alpha_mix",
                  "tolf"):
            setattr(self, k, getattr(m, k))
        self.nhist, self.maxscf, self.continuation = m.nhist, m.maxscf, bool(m.continuation)
        cp = lambda p, cnt: np.ctypeslib.as_array(p, (cnt,)).copy()
        self.H = cp(m.H, 2 * Na * Na).view(np.complex128).reshape(Na, Na, order="F")
        self.GammaL = cp(m.GammaL, 2 * Na * Na).view(np.complex128).reshape(Na, Na, order="F")
        self.GammaR = cp(m.GammaR, 2 * Na * Na).view(np.complex128).reshape(Na, Na, order="F")
        self.U_site = cp(m.U_site, Na)
        self.omega = cp(m.omega, n)
        self.model_name = m.model_name.decode()

    def __del__(self):
        if getattr(self, "_c", None):
            _host.qsah_free(self._c)
            self._c = None

    @classmethod
    def load(cls, case_dir):
        p = ctypes.POINTER(_QsahModel)()
        err = ctypes.create_string_buffer(4096)
        rc = _host.qsah_load(os.fsencode(case_dir), ctypes.byref(p), err, 4096, None)
        if rc != 0:
            raise ValueError(err.value.decode(errors="replace").strip())
        return cls(p)

    def problem(self, device=0, **over):
        """qsa_problem for this model (keeps the arrays alive on the returned object)."""
        keep = dict(H=np.asfortranarray(self.H), GammaL=np.asfortranarray(self.GammaL),
                    GammaR=np.asfortranarray(self.GammaR), U=np.ascontiguousarray(self.U_site),
                    omega=np.ascontiguousarray(self.omega))
        s = dict(alpha_mix=self.alpha_mix, tolf=self.tolf, nhist=self.nhist, maxscf=self.maxscf, order=self.order)
        s.update(over)
        p = QsaProblem(self.N_sites, s["order"], self.n_omega, _ptr(keep["H"]), _ptr(keep["GammaL"]),
                       _ptr(keep["GammaR"]), _ptr(keep["U"]), _ptr(keep["omega"]), self.mu, self.beta, self.delta,
                       s["alpha_mix"], s["tolf"], s["nhist"], s["maxscf"], device)
        p._keep = keep
        return p


class SanchoSolver:
    """One handle over a library with the qsa200.h entry points (default: the B200 library)."""

    def __init__(self, model, device=0, lib=None, prefix="qsa_", **settings):
        self.lib, self.prefix = (lib or qb._lib), prefix
        self.model = model
        self._prob = model.problem(device, **settings)
        self._h = ctypes.c_void_p()
        rc = self._f("create")(ctypes.byref(self._prob), ctypes.byref(self._h))
        if rc != 0:
            if self._h:
                self._f("destroy")(self._h)
                self._h = None
            raise qb.SolverError(f"create failed ({rc})")
        self.n_vec = int(self._f("vector_length")(self._h))

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def _check(self, rc, what):
        if rc == 0:
            return
        msg = self._f("last_error")(self._h).decode()
        if rc > 0:
            raise qb.SingularMatrixError(f"{what}: {msg}")
        raise qb.SolverError(f"{what} failed ({rc}): {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._f("destroy")(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def solve_scf(self, V, fresh_start=True):
        cap = self._prob.maxscf + 2
        log = (qb.QsScfStep * cap)()
        r = qb.QsScfResult()
        r.log, r.log_cap = log, cap
        self._check(self._f("solve_scf")(self._h, V, int(fresh_start), ctypes.byref(r)), "solve_scf")
        out = {k: getattr(r, k) for k in ("converged", "n_iter", "fmax", "aborted", "runaway", "unphysical",
                                           "i_worst", "n_worst", "w_worst", "n_resets", "seconds")}
        out["converged"] = bool(out["converged"])
        out["log"] = [(log[i].step, log[i].fmax, log[i].rms, log[i].nh) for i in range(r.n_log)]
        return out

    def current(self, V):
        J = ctypes.c_double()
        self._check(self._f("current")(self._h, V, ctypes.byref(J)), "current")
        return J.value

    def observables(self):
        m = self.model
        g = np.zeros(m.N_sites, np.complex128)
        A = np.zeros((m.N_sites, m.n_omega), np.float64, order="F")
        self._check(self._f("get_observables")(self._h, _ptr(g), _ptr(A)), "observables")
        return dict(G_less_t0=g, spectral=A)

    def initial_vector(self, V):
        x = np.zeros(self.n_vec)
        self._check(self._f("initial_vector")(self._h, V, _ptr(x)), "initial_vector")
        return x

    def residual(self, V, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        F = np.zeros_like(x)
        ab = ctypes.c_int(0)
        self._check(self._f("residual")(self._h, V, _ptr(x), _ptr(F), ctypes.byref(ab)), "residual")
        return F, bool(ab.value)

    def profile(self, enable):
        """Per-family device time (ms) and launch counts since the last call (qsa_profile)."""
        ms = np.zeros(len(KERNEL_FAMILIES))
        cnt = np.zeros(len(KERNEL_FAMILIES), np.int64)
        flag = -1 if enable is None else int(bool(enable))
        self._f("profile")(self._h, flag, _ptr(ms), _ptr(cnt), len(KERNEL_FAMILIES))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_FAMILIES)}

    def self_energies(self, x):
        """Sigma2^r, Sigma2^<, Sigma3^r, Sigma3^< as (N_sites, N_sites, n_omega) arrays."""
        m = self.model
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = [np.zeros((m.N_sites, m.N_sites, m.n_omega), np.complex128, order="F") for _ in range(4)]
        self._check(self._f("self_energies")(self._h, _ptr(x), *[_ptr(a) for a in out]), "self_energies")
        return tuple(out)


def run_program(case_dir, device=0, timeout=3600):
    """Run the SANCHO program (sancho_b200) in case_dir; returns its exit code."""
    env = dict(os.environ, QS_DEVICE=str(device))
    with open(os.path.join(case_dir, "stdout.txt"), "w") as out:
        return subprocess.run([PROGRAM, case_dir], stdout=out, stderr=subprocess.STDOUT, env=env,
                              timeout=timeout).returncode
