"""Unit pins of the oracle's building blocks against numpy (CPU only)."""
import ctypes

import numpy as np
import pytest

import oracle_lib
import quichotte_b200 as qb


def good_fft_size(nmin):
    n = nmin
    while True:
        m = n
        for r in (2, 3, 5, 7):
            while m % r == 0:
                m //= r
        if m == 1:
            return n
        n += 1


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 8, 12, 16, 21, 32, 60, 105, 672, 720, 1000, 2048, 4096, 8192, 32768])
@pytest.mark.parametrize("sign", [-1, 1])
def test_oracle_fft_matches_numpy(n, sign):
    lib = oracle_lib.lib()
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = x.copy()
    lib.qso_fft(n, y.ctypes.data_as(ctypes.c_void_p), sign)
    ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
    assert np.max(np.abs(y - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("nmin,expect", [(657, 672), (8191, 8192), (32767, 32768), (65535, 65536), (1, 1), (11, 12)])
def test_good_fft_size(nmin, expect):
    assert oracle_lib.lib().qso_good_fft_size(nmin) == expect == good_fft_size(nmin)


def test_oracle_pack_unpack_roundtrip():
    rng = np.random.default_rng(3)
    nb, Nw = 5, 7
    Gr = rng.standard_normal((nb, nb, Nw)) + 1j * rng.standard_normal((nb, nb, Nw))
    A = rng.standard_normal((nb, nb, Nw)) + 1j * rng.standard_normal((nb, nb, Nw))
    Gl = A - np.conj(A.transpose(1, 0, 2))  # anti-Hermitian
    x = qb.pack_gf(np.asfortranarray(Gr), np.asfortranarray(Gl), lib=oracle_lib.lib(), prefix="qso_")
    assert x.size == 3 * nb * nb * Nw
    R, L = qb.unpack_gf(x, nb, Nw, lib=oracle_lib.lib(), prefix="qso_")
    assert np.array_equal(R, Gr)
    assert np.allclose(L, Gl, rtol=0, atol=0)


def test_oracle_invert_matches_numpy():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((6, 9, 9)) + 1j * rng.standard_normal((6, 9, 9)) + 4 * np.eye(9)
    inv, info = qb.invert_batched(A, lib=oracle_lib.lib(), prefix="qso_")
    assert not info.any()
    assert np.allclose(inv, np.linalg.inv(A), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("single", [True, False])
def test_oracle_broyden_solves_linear_fixed_point(single):
    # x = A x + b with a contraction A: Broyden converges, the fixed point is (1-A)^-1 b
    rng = np.random.default_rng(11)
    n = 40
    A = 0.4 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    res = lambda x: (A @ x + b - x, False)
    x, conv, nit, fmax, steps = qb.broyden_solve(res, np.zeros(n), alpha_mix=0.3, nhist=8, maxscf=200, tolf=1e-12,
                                                 single_history=single, lib=oracle_lib.lib(), prefix="qso_")
    assert conv and fmax < 1e-12
    assert np.allclose(x, np.linalg.solve(np.eye(n) - A, b), atol=1e-10)
    assert steps[0][0] == 1 and len(steps) == nit
