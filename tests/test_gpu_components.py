"""Parity of each CUDA step with the oracle on the same inputs (FP64; tolerances stated
per test). Every call goes through the C ABI of libqsb200.so."""
import os

import numpy as np
import pytest

import golden_runner as g
import oracle_lib
import quichotte_b200 as qb

pytestmark = pytest.mark.gpu
CASES = os.path.join(g.GOLDEN, "cases")


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("N", [1, 2, 5, 8, 16, 18, 24, 33, 64, 100, 120, 121, 128, 136, 192, 200, 248, 256])
def test_invert_batched_matches_numpy(N):
    rng = np.random.default_rng(N)
    batch = 37
    A = rng.standard_normal((batch, N, N)) + 1j * rng.standard_normal((batch, N, N)) + 3 * np.sqrt(N) * np.eye(N)
    inv, info = qb.invert_batched(A)
    assert not info.any()
    assert rel(inv, np.linalg.inv(A)) < 1e-13  # FP64, well-conditioned


def test_invert_batched_flags_singular_matrix():
    A = np.tile(np.eye(6, dtype=np.complex128), (4, 1, 1))
    A[2, 3, :] = 0.0  # matrix 2 has a zero row
    inv, info = qb.invert_batched(A)
    assert not info[[0, 1, 3]].any()
    _, info_o = qb.invert_batched(A[2:3], lib=oracle_lib.lib(), prefix="qso_")
    assert info[2] == info_o[0] == 4  # LAPACK's zgetrf reports the same zero pivot (step 4, 1-based)
    assert np.allclose(inv[0], np.eye(6))


def test_pack_unpack_bit_exact_against_oracle():
    rng = np.random.default_rng(2)
    nb, Nw = 6, 11
    Gr = np.asfortranarray(rng.standard_normal((nb, nb, Nw)) + 1j * rng.standard_normal((nb, nb, Nw)))
    A = rng.standard_normal((nb, nb, Nw)) + 1j * rng.standard_normal((nb, nb, Nw))
    Gl = np.asfortranarray(A - np.conj(A.transpose(1, 0, 2)))
    x_gpu = qb.pack_gf(Gr, Gl)
    x_ora = qb.pack_gf(Gr, Gl, lib=oracle_lib.lib(), prefix="qso_")
    assert np.array_equal(x_gpu, x_ora)
    R, L = qb.unpack_gf(x_gpu, nb, Nw)
    R2, L2 = qb.unpack_gf(x_gpu, nb, Nw, lib=oracle_lib.lib(), prefix="qso_")
    assert np.array_equal(R, R2) and np.array_equal(L, L2)


ORDER2 = ["order2_second_order", "order2_lefthanded_siteU", "order2_dftb_blocks", "order2_dftb_hs"]


def pair(case):
    m = qb.Model.load(os.path.join(CASES, case))
    return m, qb.Solver(m), oracle_lib.solver(m)


@pytest.mark.parametrize("case", ORDER2)
def test_initial_vector_matches_oracle(case):
    m, gs, os_ = pair(case)
    assert gs.n_vec == os_.n_vec and gs.nA == os_.nA and gs.Nf == os_.Nf
    xg, xo = gs.initial_vector(m.V), os_.initial_vector(m.V)
    assert rel(xg, xo) < 1e-12


@pytest.mark.parametrize("case", ORDER2)
def test_self_energies_match_oracle(case):
    m, gs, os_ = pair(case)
    x = os_.initial_vector(m.V)
    x = x + 1e-3 * np.random.default_rng(0).standard_normal(x.size)
    SRg, SLg, S1g = gs.self_energies(x)
    SRo, SLo, S1o = os_.self_energies(x)
    assert rel(SRg, SRo) < 1e-12
    assert rel(SLg, SLo) < 1e-12
    assert np.max(np.abs(S1g - S1o)) < 1e-13


@pytest.mark.parametrize("case", ORDER2 + ["order1_hartree_fock", "order1_custom_template"])
def test_residual_matches_oracle(case):
    m, gs, os_ = pair(case)
    x = os_.initial_vector(m.V)
    Fg, ag = gs.residual(m.V, x)
    Fo, ao = os_.residual(m.V, x)
    assert ag == ao == False
    assert np.max(np.abs(Fg - Fo)) < 1e-11 * max(1.0, np.max(np.abs(x)))


# helices whose active blocks (nA = 56, 100, 120) take the tensor-core Keldysh kernel,
# including orders that are not multiples of 16 or 32
LARGE_HELICES = [(7, 4), (10, 5), (10, 6)]


@pytest.mark.parametrize("ions_turns", LARGE_HELICES)
def test_large_active_block_residual_matches_oracle(ions_turns):
    ni, nt = ions_turns
    m = qb.Model.helix(N_ions=ni, N_turns=nt, hel_length=0.34 * nt, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0,
                       lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0,
                       dw=1.0, up=1.0, delta=0.04, order=2)
    gs, os_ = qb.Solver(m), oracle_lib.solver(m)
    assert gs.nA == os_.nA == 2 * ni * nt
    xg, xo = gs.initial_vector(0.2), os_.initial_vector(0.2)
    assert rel(xg, xo) < 1e-12
    x = xo + 1e-3 * np.random.default_rng(3).standard_normal(xo.size)
    Fg, _ = gs.residual(0.2, x)
    Fo, _ = os_.residual(0.2, x)
    assert np.max(np.abs(Fg - Fo)) < 1e-11 * max(1.0, np.max(np.abs(x)))


@pytest.mark.parametrize("single", [True, False])
def test_device_broyden_matches_oracle_broyden(single):
    rng = np.random.default_rng(7)
    n = 300
    A = 0.5 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    res = lambda x: (np.tanh(A @ x) + b - x, False)
    kw = dict(alpha_mix=0.2, nhist=8, maxscf=100, tolf=1e-11, single_history=single)
    xg, cg, ng, fg, sg = qb.broyden_solve(res, np.zeros(n), **kw)
    xo, co, no, fo, so = qb.broyden_solve(res, np.zeros(n), lib=oracle_lib.lib(), prefix="qso_", **kw)
    assert cg and co and ng == no
    assert np.max(np.abs(xg - xo)) < 1e-10
    for a, b_ in zip(sg, so):
        assert a[0] == b_[0] and a[3] == b_[3]
        # two FP64 reduction orders; a single-precision history rounds each direction to
        # FP32, so its path may drift by a few FP32 ulps relative (the reference: "changes
        # the path to the fixed point, not the fixed point", common/broyden_mixing.f90:21-26)
        tol = (1e-3 * b_[1] + 1e-10) if single else (1e-6 * b_[1] + 1e-12)
        assert abs(a[1] - b_[1]) <= tol


def small_helix(delta):
    return qb.Model.helix(N_ions=3, N_turns=2, hel_length=1.0, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0,
                          lamb=0.05, U_int=0.9, GammaL_up=0.6, GammaL_down=0.4, GammaR=0.5, T=300.0, mu=0.1,
                          dw=2.0, up=2.0, delta=delta, order=2)


def radices(n):
    out = set()
    for r in (2, 3, 5, 7):
        if n % r == 0:
            out.add(r)
    return out


# energy steps chosen so that the padded FFT lengths cover radices 2, 3, 5 and 7 and both
# small and large four-step splits
DELTAS = [0.05, 0.0137, 0.0071, 0.0043, 0.0029]


@pytest.mark.parametrize("delta", DELTAS)
def test_sigma2_and_residual_match_oracle_over_fft_lengths(delta):
    m = small_helix(delta)
    gs, os_ = qb.Solver(m), oracle_lib.solver(m)
    assert gs.Nf == os_.Nf
    x = os_.initial_vector(0.3)
    x = x + 1e-3 * np.random.default_rng(1).standard_normal(x.size)
    SRg, SLg, _ = gs.self_energies(x)
    SRo, SLo, _ = os_.self_energies(x)
    assert rel(SRg, SRo) < 1e-12 and rel(SLg, SLo) < 1e-12, (m.n_omega, gs.Nf)
    Fg, _ = gs.residual(0.3, x)
    Fo, _ = os_.residual(0.3, x)
    assert np.max(np.abs(Fg - Fo)) < 1e-11 * max(1.0, np.max(np.abs(x)))


# energy steps whose padded FFT lengths are powers of two: Nf = 4096 (64 x 64), 8192
# (128 x 64), 16384 (128 x 128), 32768 (256 x 128), the specialised length-64/128/256
# transforms of both four-step stages
POW2_DELTAS = [0.0037309, 0.0018609, 0.0009293, 0.0004655]


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
@pytest.mark.parametrize("delta", POW2_DELTAS)
def test_sigma2_power_of_two_fft_lengths_match_oracle(delta, mode):
    """mode 1: autotuned; 2: the 4 x 4 tiles of the persistent kernels A and C; 3: the FP64
    forms' wide tiles (A: 2 sequences x 8 columns, C: two site pairs x 2 columns); 4: the
    4 x 2 tiles (two blocks per SM)"""
    m = small_helix(delta)
    qb.autotune(mode)
    try:
        gs, os_ = qb.Solver(m), oracle_lib.solver(m)
        assert gs.Nf == os_.Nf and gs.Nf & (gs.Nf - 1) == 0
        x = os_.initial_vector(0.3)
        x = x + 1e-3 * np.random.default_rng(2).standard_normal(x.size)
        SRg, SLg, _ = gs.self_energies(x)
        SRo, SLo, _ = os_.self_energies(x)
        assert rel(SRg, SRo) < 1e-12 and rel(SLg, SLo) < 1e-12, (m.n_omega, gs.Nf)
    finally:
        qb.autotune(1)


def test_fft_lengths_cover_all_radices():
    seen = set()
    for d in DELTAS:
        m = small_helix(d)
        seen |= radices(qb.Solver(m).Nf)
    assert seen == {2, 3, 5, 7}, seen


# ---- mixed precision (QS_PREC_MIXED) ----

MIXED_SIGMA_DELTAS = [0.05, 0.0029, 0.0037309, 0.0004655]  # Nf = 315, 5250, 4096, 32768


@pytest.mark.parametrize("delta", MIXED_SIGMA_DELTAS)
def test_mixed_sigma2_within_fp32_tolerance_of_oracle(delta):
    """FP32 transforms, 2x2 algebra and spectra: Sigma2 within 2e-5 relative of the FP64
    oracle (FP32 rounding over log2(Nf) FFT passes and the cubic products)."""
    m = small_helix(delta)
    gs, os_ = qb.Solver(m, precision=qb.QS_PREC_MIXED), oracle_lib.solver(m)
    x = os_.initial_vector(0.3)
    x = x + 1e-3 * np.random.default_rng(4).standard_normal(x.size)
    SRg, SLg, _ = gs.self_energies(x)
    SRo, SLo, _ = os_.self_energies(x)
    assert rel(SRg, SRo) < 2e-5 and rel(SLg, SLo) < 2e-5, (rel(SRg, SRo), rel(SLg, SLo))
    assert rel(SRg, SRo) > 1e-12  # the FP32 path ran


def large_helix(ni, nt, delta=0.04):
    return qb.Model.helix(N_ions=ni, N_turns=nt, hel_length=0.34 * nt, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0,
                          lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0,
                          dw=1.0, up=1.0, delta=delta, order=2)


@pytest.mark.parametrize("ions_turns", LARGE_HELICES)
def test_mixed_sigma2_rounding_is_relative_to_the_largest_spectrum(ions_turns):
    """On the large helices |Sigma^r| reaches 10^3-10^4 times |Sigma^<| (sharp resonances on
    the grid); the FP32 transforms round relative to the largest spectra they carry, so
    both self-energies are within 2e-6 of the oracle relative to max |Sigma^r| (measured:
    Sigma^r 3e-7 relative to itself, Sigma^< 2e-8 of max |Sigma^r| at nA = 100)."""
    m = large_helix(*ions_turns)
    gs, os_ = qb.Solver(m, precision=qb.QS_PREC_MIXED), oracle_lib.solver(m)
    x = os_.initial_vector(0.2) + 1e-3 * np.random.default_rng(6).standard_normal(gs.n_vec)
    SRg, SLg, _ = gs.self_energies(x)
    SRo, SLo, _ = os_.self_energies(x)
    scale = np.max(np.abs(SRo))
    assert np.max(np.abs(SRg - SRo)) / scale < 2e-6
    assert np.max(np.abs(SLg - SLo)) / scale < 2e-6
    assert np.max(np.abs(SRg - SRo)) / scale > 1e-12  # the FP32 path ran


@pytest.mark.parametrize("ions_turns", [(4, 2)] + LARGE_HELICES)
def test_mixed_residual_tensor_core_keldysh_matches_oracle(ions_turns):
    """The FP32-phase residual of a mixed handle with the Keldysh products forced onto the
    3xTF32 tensor-core kernel (tcgen05, FP32 accumulation in tensor memory). Its G^r part
    is the FP64 Dyson inverse of the FP32 self-energies, so its error is that rounding times
    the conditioning of the Dyson matrices: 2e-5 of max|G_out| at nA = 16, up to ~1e-2 at
    nA = 120 (delta = 0.04, sharp resonances). The tensor-core products add no error of
    their own beyond it: the G^< part's error stays within 3x the G^r part's (+1e-5)."""
    ni, nt = ions_turns
    m = large_helix(ni, nt)
    qb.autotune(-1)
    qb.autotune(2)  # the first candidate of every decision: the 3xTF32 kernel in the FP32 phase
    try:
        gs, os_ = qb.Solver(m, precision=qb.QS_PREC_MIXED), oracle_lib.solver(m)
        x = os_.initial_vector(0.2) + 1e-3 * np.random.default_rng(6).standard_normal(gs.n_vec)
        Fg, ag = gs.residual(0.2, x)
    finally:
        qb.autotune(1)
    Fo, ao = os_.residual(0.2, x)
    assert not ag and not ao
    nA = gs.nA
    blk = 3 * nA * nA
    Fg, Fo, G = Fg.reshape(-1, blk), Fo.reshape(-1, blk), (Fo + x).reshape(-1, blk)
    scale = np.max(np.abs(G))
    r = 2 * nA * nA  # pack_gf block: Re, Im G^r, then G^<
    err_r = np.max(np.abs(Fg[:, :r] - Fo[:, :r])) / scale
    err_l = np.max(np.abs(Fg[:, r:] - Fo[:, r:])) / scale
    assert 1e-12 < max(err_r, err_l)  # not the FP64 path
    if nA <= 16:
        assert max(err_r, err_l) < 2e-5, (err_r, err_l)
    else:
        assert err_r < 5e-2, err_r
    assert err_l <= 3 * err_r + 1e-5, (err_r, err_l)


@pytest.mark.parametrize("case", ORDER2)
def test_mixed_solve_matches_fp64_solve(case):
    """A mixed solve converges on FP64 residuals: currents, occupations and the spectral
    function agree with the plain FP64 solve to far better than 1e-6 relative."""
    m = qb.Model.load(os.path.join(CASES, case))
    f64, mix = qb.Solver(m), qb.Solver(m, precision=qb.QS_PREC_MIXED)
    r64, rmx = f64.solve_scf(m.V), mix.solve_scf(m.V)
    assert r64["converged"] and rmx["converged"]
    assert rmx["n_mixed"] > 0 and r64["n_mixed"] == 0
    j64, jmx = np.array(f64.current(m.V)), np.array(mix.current(m.V))
    assert np.max(np.abs(jmx - j64)) <= 1e-6 * np.max(np.abs(j64)), (j64, jmx)
    o64, omx = f64.observables(), mix.observables()
    for k in o64:
        a, b_ = np.asarray(omx[k]), np.asarray(o64[k])
        assert np.max(np.abs(a - b_)) <= 1e-6 * max(np.max(np.abs(b_)), 1e-300), k


# ---- autotuner: every variant it chooses between computes the same step ----

@pytest.mark.parametrize("mode", [2, 3, 4])
@pytest.mark.parametrize("ions_turns", [(4, 2), (7, 4), (10, 6)])
def test_forced_kernel_variants_match_oracle(mode, ions_turns):
    """Blocked/tensor-core (mode 2), unblocked/CUDA-core (mode 3) and the blocked Dyson on the
    global workspace with two blocks per SM (mode 4, N > 16) at N = nA = 16, 56, 120:
    residual within 1e-11 of the oracle."""
    ni, nt = ions_turns
    m = qb.Model.helix(N_ions=ni, N_turns=nt, hel_length=0.34 * nt, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0,
                       lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0,
                       dw=1.0, up=1.0, delta=0.04, order=2)
    qb.autotune(mode)
    try:
        gs, os_ = qb.Solver(m), oracle_lib.solver(m)
        x = os_.initial_vector(0.2) + 1e-3 * np.random.default_rng(5).standard_normal(gs.n_vec)
        Fg, _ = gs.residual(0.2, x)
        Fo, _ = os_.residual(0.2, x)
        assert np.max(np.abs(Fg - Fo)) < 1e-11 * max(1.0, np.max(np.abs(x)))
    finally:
        qb.autotune(1)


@pytest.mark.parametrize("mode", [2, 3, 4])
@pytest.mark.parametrize("ions_turns", [(17, 4), (16, 6)])
def test_dyson_above_shared_memory_matches_oracle(mode, ions_turns):
    """N = 136, 192: the matrix no longer fits in shared memory. Mode 2 forces the blocked
    tensor-core Gauss-Jordan on the global workspace, mode 3 the unblocked one; the residual
    within 1e-11 of the oracle either way."""
    ni, nt = ions_turns
    m = qb.Model.helix(N_ions=ni, N_turns=nt, hel_length=0.34 * nt, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0,
                       lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0,
                       dw=1.0, up=1.0, delta=0.08, order=2)
    qb.autotune(mode)
    try:
        gs, os_ = qb.Solver(m), oracle_lib.solver(m)
        assert gs.nA == 2 * ni * nt
        x = os_.initial_vector(0.2) + 1e-3 * np.random.default_rng(8).standard_normal(gs.n_vec)
        Fg, _ = gs.residual(0.2, x)
        Fo, _ = os_.residual(0.2, x)
        assert np.max(np.abs(Fg - Fo)) < 1e-11 * max(1.0, np.max(np.abs(x)))
    finally:
        qb.autotune(1)


def test_autotuner_records_a_choice_per_size():
    m = qb.Model.helix(N_ions=7, N_turns=4, hel_length=1.36, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0,
                       lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0,
                       dw=1.0, up=1.0, delta=0.04, order=2)
    qb.autotune(-1)
    qb.autotune(1)
    s = qb.Solver(m)
    s.residual(0.3, s.initial_vector(0.3))
    assert s.nA == 56
    key = qb.tune_key(56, m.n_omega)
    assert qb.tuned_choice(qb.TUNE_DYSON, key) in (1, 2, 3) and qb.tuned_choice(qb.TUNE_KELDYSH, key) in (1, 2)
    s.close()
    # the FP32 phase of a mixed handle tunes its own Keldysh decision among the 3xTF32
    # tensor-core kernel (3) and the FP64 ones (1, 2)
    mx = qb.Solver(m, precision=qb.QS_PREC_MIXED)
    mx.residual(0.3, mx.initial_vector(0.3))
    assert qb.tuned_choice(qb.TUNE_KELDYSH32, key) in (1, 2, 3)
    mx.close()


# ---- failure detection: SCF runaway, as scf_residual2 + check_diag_sanity ----

@pytest.mark.parametrize("ions", [3, 4])
@pytest.mark.parametrize("stride", [7, 1])
def test_runaway_state_aborts_like_the_oracle(stride, ions):
    """A state holding NaNs (every 7th entry, or all) makes the residual report abort
    (src/scf.f90:180-186 via the NaN test of common/scf_checks.f90:59-91) and zero F, on the
    GPU as in the oracle. The Dyson kernels keep every pivot row in range for NaN columns,
    and a normal residual follows on the same handle. N = 12 takes the unblocked Gauss-Jordan
    kernel, N = 16 the blocked one."""
    m = small_helix(0.05) if ions == 3 else qb.Model.helix(
        N_ions=4, N_turns=2, hel_length=0.6, hel_radius=0.7, hand=1.0, E_CC=0.0, t_hop=1.0, lamb=0.01, U_int=1.0,
        GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0, dw=1.0, up=1.0, delta=0.04, order=2)
    gs, os_ = qb.Solver(m), oracle_lib.solver(m)
    x0 = os_.initial_vector(0.3)
    x = x0.copy()
    x[::stride] = np.nan
    Fg, ag = gs.residual(0.3, x)
    Fo, ao = os_.residual(0.3, x)
    assert ag and ao
    assert not np.any(Fg) and not np.any(Fo)
    Fg2, ag2 = gs.residual(0.3, x0)
    Fo2, _ = os_.residual(0.3, x0)
    assert not ag2 and np.max(np.abs(Fg2 - Fo2)) < 1e-11
