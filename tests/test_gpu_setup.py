"""The set-up's dense linear algebra on the device against LAPACK (numpy) restatements.

- qs_hermitian_eigensystem (and qs_hermitian_eigenvalues, without vectors) replace
  hermitian_eigensystem (common/linear_algebra.f90:32-56,
  zheev): eigenvalues within 1e-12 ||A||_2 of numpy.linalg.eigh (LAPACK), eigenvectors by
  their residual ||A Z - Z E|| and orthonormality (a degenerate eigenvalue's basis is not
  unique, so the subspace projector is compared instead of the vectors).
- qs_dftb_lowdin replaces the dense part of build_hamiltonian_from_dftb_hs
  (src/hamiltonian.f90:625-689): H within 1e-12 (relative to max |H|) of the same formulas in
  numpy, both SOC forms; a non-positive-definite overlap is refused as the reference stops.
- The program's own use of both is covered by the golden cases (test_gpu_scf), whose
  order2_dftb_hs case compares hamiltonian_matrix.dat.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

qb = pytest.importorskip("quichotte_b200")

TOL = 1e-12


def _herm(rng, N, scale=1.0):
    X = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    return scale * (X + X.conj().T) / 2


def _check_eigensystem(A, E, Z, tol=TOL):
    N = A.shape[0]
    En = np.linalg.eigvalsh(A)
    nrm = max(1.0, np.max(np.abs(En)))
    assert np.all(np.diff(E) >= 0), "eigenvalues not ascending"
    assert np.max(np.abs(E - En)) <= tol * nrm, np.max(np.abs(E - En))
    assert np.max(np.abs(A @ Z - Z * E)) <= 10 * tol * nrm
    assert np.max(np.abs(Z.conj().T @ Z - np.eye(N))) <= 10 * tol


@pytest.mark.parametrize("N", [1, 2, 3, 16, 17, 64, 120, 129, 248])
def test_eigensystem_random_batch(N):
    rng = np.random.default_rng(100 + N)
    A = np.stack([_herm(rng, N, s) for s in (1.0, 1e-3, 50.0)])
    E, Z, info = qb.hermitian_eigensystem(A)
    assert list(info) == [0, 0, 0]
    for b in range(3):
        _check_eigensystem(A[b], E[b], Z[b])


def test_eigensystem_helix_kramers_pairs():
    # the 120x120 helix with SOC: time reversal makes every level twofold
    m = qb.Model.helix(N_ions=10, N_turns=6, hel_length=0.34 * 6 * 9 / 10, hel_radius=0.7, hand=1.0, E_CC=0.0,
                       t_hop=1.0, lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0,
                       mu=0.0, dw=2.0, up=2.0, delta=0.01)
    E, Z, info = qb.hermitian_eigensystem(m.H)
    assert info == 0
    _check_eigensystem(m.H, E, Z)
    En, Zn = np.linalg.eigh(m.H)
    # projectors onto each Kramers pair agree
    for k in range(0, m.Norb, 2):
        P = Z[:, k:k + 2] @ Z[:, k:k + 2].conj().T
        Pn = Zn[:, k:k + 2] @ Zn[:, k:k + 2].conj().T
        assert np.max(np.abs(P - Pn)) < 1e-9


def test_eigensystem_edge_cases():
    N = 7
    zero = np.zeros((N, N), complex)
    diag = np.diag([3.0, -1.0, 2.0, -1.0, 0.5, 7.0, -4.0]).astype(complex)
    ident = 2.5 * np.eye(N, dtype=complex)
    nan = _herm(np.random.default_rng(5), N)
    nan[2, 4] = np.nan
    nan[4, 2] = np.nan
    ok = _herm(np.random.default_rng(6), N)
    E, Z, info = qb.hermitian_eigensystem(np.stack([zero, diag, ident, nan, ok]))
    assert list(info) == [0, 0, 0, 1, 0]
    assert np.all(E[0] == 0) and np.array_equal(Z[0], np.eye(N))
    # an already diagonal matrix: sorted diagonal (ties in index order), permutation vectors
    order = np.argsort(np.diag(diag).real, kind="stable")
    assert np.array_equal(E[1], np.diag(diag).real[order])
    assert np.array_equal(Z[1], np.eye(N)[:, order])
    assert np.all(E[2] == 2.5)
    _check_eigensystem(ok, E[4], Z[4])
    with pytest.raises(qb.SolverError):
        qb.hermitian_eigensystem(np.zeros((2049, 2049), complex))


def test_eigensystem_two_calls_same_result():
    rng = np.random.default_rng(11)
    A = _herm(rng, 48)
    E1, Z1, _ = qb.hermitian_eigensystem(A)
    E2, Z2, _ = qb.hermitian_eigensystem(A)
    assert np.array_equal(E1, E2) and np.array_equal(Z1, Z2)


def _lowdin_numpy(S, H0, Lam, dual):
    """src/hamiltonian.f90:625-689 in numpy (LAPACK eigh for dsyev)."""
    ev, U = np.linalg.eigh(S)
    W = U / np.sqrt(np.sqrt(ev))
    Smh = W @ W.T
    I2 = np.eye(2)
    Sx2, Sm2, Hao = np.kron(S, I2), np.kron(Smh, I2), np.kron(H0, I2).astype(complex)
    Hao = Hao + (0.5 * (Sx2 @ Lam + Lam @ Sx2) if dual else Lam)
    H = Sm2 @ Hao @ Sm2
    return 0.5 * (H + H.conj().T), ev.min()


# N <= 160: S^-1/2 by Newton-Schulz on the eigenvalues of one block; above: the Jacobi eigenpairs.
# spread = ||S - I||_2 (0.99: condition number ~200, 13 Newton-Schulz steps; 0: S = I)
@pytest.mark.parametrize("N,dual,spread", [(1, True, 0.1), (9, True, 0.1), (31, False, 0.1), (124, True, 0.1),
                                           (80, True, 0.99), (5, False, 0.0), (200, True, 0.1)])
def test_dftb_lowdin_matches_numpy(N, dual, spread):
    rng = np.random.default_rng(7 + N)
    P = rng.standard_normal((N, N))
    P = 0.5 * (P + P.T)
    S = np.eye(N) + spread * P / max(1e-300, np.linalg.norm(P, 2))
    H0 = rng.standard_normal((N, N))
    H0 = 0.5 * (H0 + H0.T) * 27.211386245988
    Lam = 0.01 * _herm(rng, 2 * N)
    H, evmin = qb.dftb_lowdin(S, H0, Lam, dual)
    Hn, evn = _lowdin_numpy(S, H0, Lam, dual)
    assert abs(evmin - evn) <= 1e-13
    assert np.max(np.abs(H - Hn)) <= TOL * np.max(np.abs(Hn))
    assert np.array_equal(H, H.conj().T)


def test_dftb_lowdin_refuses_indefinite_overlap():
    N = 6
    S = np.eye(N)
    S[0, 1] = S[1, 0] = 1.5  # eigenvalues 1 +- 1.5
    with pytest.raises(qb.SolverError, match="not positive definite"):
        qb.dftb_lowdin(S, np.zeros((N, N)), np.zeros((2 * N, 2 * N), complex))


@pytest.mark.parametrize("N", [1, 2, 3, 16, 17, 64, 120, 129, 160, 161, 248])
def test_eigenvalues_only_random_batch(N):
    # N <= 160: one block per matrix with the matrix in shared memory; above: the sweep graphs
    rng = np.random.default_rng(300 + N)
    A = np.stack([_herm(rng, N, s) for s in (1.0, 1e-3, 50.0)])
    A0 = A.copy()
    E, info = qb.hermitian_eigenvalues(A)
    assert list(info) == [0, 0, 0]
    assert np.array_equal(A, A0)
    for b in range(3):
        En = np.linalg.eigvalsh(A[b])
        assert np.all(np.diff(E[b]) >= 0)
        assert np.max(np.abs(E[b] - En)) <= TOL * max(1.0, np.max(np.abs(En)))


def test_eigenvalues_only_edge_cases_and_helix():
    N = 7
    diag = np.diag([3.0, -1.0, 2.0, -1.0, 0.5, 7.0, -4.0]).astype(complex)
    nan = _herm(np.random.default_rng(9), N)
    nan[1, 5] = np.nan
    nan[5, 1] = np.nan
    ok = _herm(np.random.default_rng(10), N)
    E, info = qb.hermitian_eigenvalues(np.stack([np.zeros((N, N), complex), diag, nan, ok]))
    assert list(info) == [0, 0, 1, 0]
    assert np.all(E[0] == 0)
    assert np.array_equal(E[1], np.sort(np.diag(diag).real))
    assert np.max(np.abs(E[3] - np.linalg.eigvalsh(ok))) <= TOL * np.max(np.abs(E[3]))
    m = qb.Model.helix(N_ions=10, N_turns=6, hel_length=0.34 * 6 * 9 / 10, hel_radius=0.7, hand=1.0, E_CC=0.0,
                       t_hop=1.0, lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0,
                       mu=0.0, dw=2.0, up=2.0, delta=0.01)
    Eh, infoh = qb.hermitian_eigenvalues(m.H)
    assert infoh == 0
    assert np.max(np.abs(Eh - np.linalg.eigvalsh(m.H))) <= TOL * np.max(np.abs(Eh))
    assert np.max(np.abs(Eh - m.Ev)) <= TOL * np.max(np.abs(Eh))  # the host's Jacobi


@pytest.mark.parametrize("scale", [1e250, 1e-250])
def test_extreme_scales_as_lapack(scale):
    # |a|^2 would overflow (or underflow) in the convergence test: both paths scale the
    # matrix by an exact power of two first, as LAPACK does
    rng = np.random.default_rng(21)
    A = np.stack([_herm(rng, N=40, scale=scale), _herm(rng, N=40, scale=scale)])
    En = np.linalg.eigvalsh(A)
    E1, Z, info1 = qb.hermitian_eigensystem(A)
    E2, info2 = qb.hermitian_eigenvalues(A)
    assert list(info1) == [0, 0] and list(info2) == [0, 0]
    for b in range(2):
        nrm = np.max(np.abs(En[b]))
        assert np.max(np.abs(E1[b] - En[b])) <= TOL * nrm
        assert np.max(np.abs(E2[b] - En[b])) <= TOL * nrm
        assert np.max(np.abs(Z[b].conj().T @ Z[b] - np.eye(40))) <= 10 * TOL
