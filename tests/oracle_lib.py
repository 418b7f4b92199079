"""Test-side access to the CPU oracle (oracle/_build), the checker of the B200 solver."""
import ctypes
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle", "_build")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
ORACLE_EXE = os.path.join(ORACLE_DIR, "quichotte_oracle")
SANCHO_ORACLE_EXE = os.path.join(ORACLE_DIR, "sancho_oracle")

_lib = None


def lib():
    global _lib
    if _lib is None:
        import quichotte_b200 as qb  # loads the host layer (RTLD_GLOBAL) the oracle program also uses
        _lib = ctypes.CDLL(ORACLE_LIB)
        qb.bind_solver(_lib, "qso_")
        _lib.qso_fft.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        _lib.qso_good_fft_size.argtypes = [ctypes.c_int]
    return _lib


def sancho_lib():
    """The oracle library with the qsa200.h signatures on its qsao_* entry points."""
    import sancho_b200 as sb
    sb.bind_solver(lib(), "qsao_")
    return lib()


def sancho_solver(model, **kw):
    import sancho_b200 as sb
    return sb.SanchoSolver(model, lib=sancho_lib(), prefix="qsao_", **kw)


def solver(model, **kw):
    import quichotte_b200 as qb
    return qb.Solver(model, lib=lib(), prefix="qso_", **kw)
