"""The serving loop (qs_server_*): HBM admission, concurrent solves, and results that do
not depend on what else is in flight. Every call goes through the C ABI of libqsb200.so."""
import numpy as np
import pytest

import quichotte_b200 as qb

pytestmark = pytest.mark.gpu


def helix(ions, turns, U, delta):
    return qb.Model.helix(N_ions=ions, N_turns=turns, hel_length=0.34 * turns * (ions - 1) / ions, hel_radius=0.7,
                          hand=1.0, E_CC=0.0, t_hop=1.0, lamb=0.01, U_int=U, GammaL_up=0.5, GammaL_down=0.5,
                          GammaR=0.5, T=300.0, mu=0.0, dw=1.0, up=1.0, delta=delta, order=2)


# (sites/turn, turns, U, delta, V): different active blocks (12..48) and grids (n ~ 150..700)
REQUESTS = [(3, 2, 0.5, 0.02, 0.3), (4, 2, 1.0, 0.03, -0.5), (5, 3, 0.8, 0.015, 0.1), (3, 4, 1.2, 0.025, 0.9),
            (6, 2, 0.4, 0.02, -0.2), (4, 3, 1.5, 0.012, 0.6), (6, 4, 0.7, 0.03, -0.8), (3, 1, 0.9, 0.01, 0.0)]
SETTINGS = dict(alpha_mix=0.5, nhist=8, tolf=1e-7, maxscf=200, single_history=1)


def test_estimate_covers_what_a_handle_allocates():
    for ions, turns, U, delta, V in REQUESTS[:4]:
        m = helix(ions, turns, U, delta)
        est = qb.estimate_gib(m, **SETTINGS)
        s = qb.Solver(m, **SETTINGS)
        got = s.device_gib()
        s.close()
        assert got <= est <= 1.25 * got + 0.01, (ions, turns, got, est)


def test_server_results_match_stand_alone_solves_bit_for_bit():
    models = [helix(i, t, U, d) for i, t, U, d, _ in REQUESTS]
    alone = []
    for m, (_, _, _, _, V) in zip(models, REQUESTS):
        s = qb.Solver(m, **SETTINGS)
        r = s.solve_scf(V, fresh_start=True)
        alone.append((r["converged"], r["n_iter"], s.current(V)))
        s.close()
    srv = qb.Server(max_inflight=4)
    for k, (m, req) in enumerate(zip(models, REQUESTS)):
        assert srv.submit(m, req[4], k, **SETTINGS) == 0
    res = {r["id"]: r for r in srv.drain()}
    srv.close()
    assert sorted(res) == list(range(len(REQUESTS)))
    for k, (conv, nit, (ju, jd)) in enumerate(alone):
        r = res[k]
        assert r["status"] == 0 and bool(r["converged"]) == conv and r["n_iter"] == nit, (k, r, nit)
        # the same kernels, deterministic reductions, a handle and stream of its own
        assert r["J_up"] == ju and r["J_down"] == jd, (k, r["J_up"], ju, r["J_down"], jd)
    # the solves overlapped: some request started before an earlier-admitted one finished
    spans = sorted((r["t_start"], r["t_done"]) for r in res.values())
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_server_admission_keeps_the_budget():
    models = [helix(i, t, U, d) for i, t, U, d, _ in REQUESTS]
    est = [qb.estimate_gib(m, **SETTINGS) + 0.5 for m in models]
    budget = 2.2 * max(est)
    srv = qb.Server(max_inflight=8, hbm_budget_gib=budget)
    for k, (m, req) in enumerate(zip(models, REQUESTS)):
        assert srv.submit(m, req[4], k, **SETTINGS) == 0
    res = srv.drain()
    srv.close()
    assert len(res) == len(REQUESTS) and all(r["status"] == 0 for r in res)
    # at every admission instant the admitted memory stays within the budget
    for r in res:
        t = r["t_start"]
        live = sum(q["device_gib"] for q in res if q["t_start"] <= t < q["t_done"])
        assert live <= budget + 1e-9, (t, live, budget)


def test_server_refuses_a_request_larger_than_the_budget():
    m = helix(6, 4, 0.7, 0.03)
    srv = qb.Server(max_inflight=2, hbm_budget_gib=0.05)
    assert srv.submit(m, 0.1, 0, **SETTINGS) == qb.QS_ERR_TOO_LARGE
    assert srv.pending() == 0
    srv.close()
