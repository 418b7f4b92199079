"""End-to-end parity of the CUDA SCF with the oracle and with the reference's golden files.

- Golden: the quichotte_b200 program on every case of the reference's regression suite,
  compared as the reference's runner does (1e-6 abs + 1e-5 rel, tests/run_tests.f90:14).
- Oracle, tight: solve_scf with tolf = 1e-12 and a double-precision Broyden history, so
  both sides converge onto the same fixed point; currents, occupations (G_less_obs) and
  the spectral function (dosd) must agree to 1e-10 relative (plain FP64 target).
"""
import os

import numpy as np
import pytest

import golden_runner as g
import oracle_lib
import quichotte_b200 as qb

pytestmark = pytest.mark.gpu
CASES = g.cases()


@pytest.mark.parametrize("case,rc,refs", CASES, ids=[c[0] for c in CASES])
def test_program_reproduces_reference_case(case, rc, refs, workdir):
    ok, worst, msg, work = g.check_case(qb.PROGRAM, case, rc, refs, os.path.join(workdir, "gpu"))
    assert ok, msg


TIGHT = ["order2_second_order", "order2_lefthanded_siteU", "order2_dftb_hs", "order2_dftb_blocks",
         "order1_hartree_fock", "order0_noninteracting", "order0_dftb_blocks"]


@pytest.mark.parametrize("case", TIGHT)
def test_solve_scf_matches_oracle_to_1e10(case):
    m = qb.Model.load(os.path.join(g.GOLDEN, "cases", case))
    kw = dict(tolf=1e-12, tolf_order1=1e-13, single_history=0, maxscf=400)
    gs, os_ = qb.Solver(m, **kw), oracle_lib.solver(m, **kw)
    for k, V in enumerate([m.V, m.V + m.delv]):
        rg, ro = gs.solve_scf(V, k == 0), os_.solve_scf(V, k == 0)
        assert rg["converged"] and ro["converged"]
        Jg, Jo = np.array(gs.current(V)), np.array(os_.current(V))
        assert np.all(np.abs(Jg - Jo) <= 1e-10 * np.abs(Jo) + 1e-14), (Jg, Jo)
        og, oo = gs.observables(), os_.observables()
        for key in ("G_less_obs", "dosd"):
            err = np.max(np.abs(og[key] - oo[key])) / np.max(np.abs(oo[key]))
            assert err < 1e-10, (key, err)


@pytest.mark.parametrize("case", ["order2_second_order", "order2_dftb_hs"])
def test_graph_replayed_residuals_equal_eager_ones(case):
    """The FP64 Broyden loop replays each residual's launches from a CUDA graph (captured once
    per (x, F, V) buffer pair). The same sweep with per-launch profiling on runs every launch
    eagerly: both take the same steps and give bit-identical currents and observables, and
    both count the same kernel launches."""
    m = qb.Model.load(os.path.join(g.GOLDEN, "cases", case))
    a, b = qb.Solver(m), qb.Solver(m)
    b.profile(True)
    for k, V in enumerate([m.V, m.V + 0.1]):
        l0 = qb.kernel_launches()
        ra = a.solve_scf(V, k == 0)
        la = qb.kernel_launches() - l0
        l0 = qb.kernel_launches()
        rb = b.solve_scf(V, k == 0)
        lb = qb.kernel_launches() - l0
        assert (ra["converged"], ra["n_iter"]) == (rb["converged"], rb["n_iter"])
        assert la == lb
        assert a.current(V) == b.current(V)
        oa, ob = a.observables(), b.observables()
        for key in oa:
            assert np.array_equal(oa[key], ob[key]), key
    assert a.graph_replays() > 0 and b.graph_replays() == 0
