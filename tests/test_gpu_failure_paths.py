"""Failure paths of the SCF against the oracle, driven from the host (no GPU fault):

- final_sanity (src/scf.f90:260-275, check_diag_sanity common/scf_checks.f90:59-91): an
  energy window that holds only part of the spectrum leaves some states with less than half
  of their spectral weight. solve_scf then reports "CONVERGED TO AN UNPHYSICAL SOLUTION"
  (src/scf.f90:142-150): converged = .false., with the worst state's index, occupation and
  spectral weight. The GPU must flag the same state with the same numbers.
- the Broyden history reset (common/broyden_mixing.f90:155-162): the history is dropped
  when dposv reports a non-positive pivot. With finite residuals w0^2 I + dF^T dF is
  positive definite, so the branch needs a non-finite residual. The reference links
  OpenBLAS, whose dpotrf fails only on a pivot <= 0: a residual that returns an infinite
  component makes dF and the Gram column NaN, dposv passes the NaN on to gamma instead of
  failing, and the mixed x turns NaN for good. Both sides must take that same path (same
  history lengths and max|F| per step, no reset, no convergence).
"""
import os

import numpy as np
import pytest

import golden_runner as g
import oracle_lib
import quichotte_b200 as qb

pytestmark = pytest.mark.gpu
CASES = os.path.join(g.GOLDEN, "cases")


def windowed(case, lo, hi, order=None):
    """The case's model with its energy grid cut to lo < omega < hi (same spacing)."""
    m = qb.Model.load(os.path.join(CASES, case))
    keep = (m.omega > lo) & (m.omega < hi)
    m.omega = np.ascontiguousarray(m.omega[keep])
    m.n_omega = int(m.omega.size)
    assert m.n_omega > 16, m.n_omega
    if order is not None:
        m.order = order
    return m


def state_sums(obs, delta):
    """Per-state occupation n_i and spectral weight w_i as check_diag_sanity forms them."""
    n = np.imag(np.diag(obs["G_less_obs"]))
    w = -(delta / np.pi) * np.sum(obs["dosd"], axis=1)
    return n, w


@pytest.mark.parametrize("case,order,window", [
    ("order0_dftb_blocks", 0, (0.2, 40.0)),
    ("order0_noninteracting", 0, (2.3, 40.0)),
    ("order2_lefthanded_siteU", 2, (2.2, 40.0)),
])
def test_unphysical_solution_reported_like_the_oracle(case, order, window):
    m = windowed(case, *window, order=order)
    kw = dict(tolf=1e-11, tolf_order1=1e-12, single_history=0, maxscf=400)
    gs, os_ = qb.Solver(m, **kw), oracle_lib.solver(m, **kw)
    rg, ro = gs.solve_scf(m.V, True), os_.solve_scf(m.V, True)
    # the oracle drives the branch: the SCF itself converged, the final sweep is unphysical
    assert ro["unphysical"] and not ro["converged"] and not ro["aborted"]
    n, w = state_sums(os_.observables(), m.delta)
    assert np.min(w) < 0.5
    # no near-tie among the candidates, so the worst state is well defined at 1e-10
    dev = np.sort(np.abs(n - 0.5))
    assert len(dev) < 2 or dev[-1] - dev[-2] > 1e-8 or np.sort(w)[1] - np.sort(w)[0] > 1e-8
    assert rg["unphysical"] == ro["unphysical"] and rg["runaway"] == ro["runaway"]
    assert rg["converged"] == ro["converged"] and rg["aborted"] == ro["aborted"]
    assert rg["i_worst"] == ro["i_worst"], (rg["i_worst"], ro["i_worst"])
    assert abs(rg["n_worst"] - ro["n_worst"]) <= 1e-10 * max(1.0, abs(ro["n_worst"]))
    assert abs(rg["w_worst"] - ro["w_worst"]) <= 1e-10 * max(1.0, abs(ro["w_worst"]))
    if order > 0:
        assert rg["n_iter"] == ro["n_iter"]


@pytest.mark.parametrize("single", [True, False])
def test_broyden_nonfinite_gram_matches_oracle(single):
    rng = np.random.default_rng(11)
    n = 257
    A = 0.4 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)

    def make_residual():
        calls = {"k": 0}

        def res(x):
            calls["k"] += 1
            xs = np.where(np.isfinite(x), x, 0.0)
            F = np.tanh(A @ xs) + b - xs
            if calls["k"] == 4:
                F[17] = np.inf  # one infinite component at step 4
            return F, False
        return res

    kw = dict(alpha_mix=0.3, nhist=6, maxscf=40, tolf=1e-11, single_history=single)
    xg, cg, ng, fg, sg = qb.broyden_solve(make_residual(), np.zeros(n), **kw)
    xo, co, no, fo, so = qb.broyden_solve(make_residual(), np.zeros(n), lib=oracle_lib.lib(), prefix="qso_", **kw)
    assert not cg and not co and ng == no == 40
    assert [s[3] for s in sg] == [s[3] for s in so]  # history lengths: no reset on either side
    for a, b_ in zip(sg, so):
        assert a[1] == b_[1] or abs(a[1] - b_[1]) <= 1e-12 * abs(b_[1]), (a, b_)
    assert np.isnan(xg).all() and np.isnan(xo).all()
