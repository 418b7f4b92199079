"""SANCHO on B200 (include/qsa200.h) against the CPU oracle's restatement of SANCHO/src and
against SANCHO's own regression suite (SANCHO/tests, copied under tests/golden/sancho).

Parity bars: the bubble sums and self-energies (src/self_energies.f90:49-207) and the SCF
residual (src/scf.f90:102-195) within 1e-11 of the oracle relative to the largest element
(FP64, the summation order of the step-3 convolutions differs); solves with the same
Broyden steps, convergence flags and currents to 1e-9; the program's output files within
the reference runner's 1e-6 abs + 1e-5 rel (tests/run_tests.f90:14)."""
import os
import re
import shutil

import numpy as np
import pytest

import golden_runner as g
import oracle_lib

pytestmark = pytest.mark.gpu

sb = pytest.importorskip("sancho_b200")

BASE = os.path.join(g.GOLDEN_SANCHO, "cases", "order2_second_order", "input.dat")


def case_dir(tmp, name, **keys):
    """A SANCHO input.dat: the order-2 regression case with `keys` replaced or added."""
    d = os.path.join(tmp, name)
    os.makedirs(d, exist_ok=True)
    text = open(BASE).read()
    for k, v in keys.items():
        pat = re.compile(rf"^{k}\s*=.*$", re.M)
        line = f"{k} = {v}"
        text = pat.sub(line, text) if pat.search(text) else text + line + "\n"
    open(os.path.join(d, "input.dat"), "w").write(text)
    return d


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# (name, overrides): the regression chain at orders 0-3, a longer chain on a finer grid (n not
# a multiple of the 128-wide tiles, several tiles per sum), a single site, asymmetric U
MODELS = [
    ("o0", dict(order=0)),
    ("o1", dict(order=1)),
    ("o2", dict(order=2)),
    ("o3", dict(order=3)),
    ("o3_long", dict(order=3, N_sites=7, delta=0.004, U_int=1.1)),
    ("o2_single_site", dict(order=2, N_sites=1)),
    ("o2_wide", dict(order=2, N_sites=12, delta=0.006)),
]


@pytest.fixture(scope="module")
def models(tmp_path_factory):
    tmp = str(tmp_path_factory.mktemp("sancho"))
    return {name: sb.SanchoModel.load(case_dir(tmp, name, **kw)) for name, kw in MODELS}


def noisy_input(o, V, seed):
    x = o.initial_vector(V)
    return x + 1e-3 * np.random.default_rng(seed).standard_normal(x.size) * np.max(np.abs(x))


@pytest.mark.parametrize("name", ["o2", "o3", "o3_long", "o2_single_site", "o2_wide"])
def test_self_energies_match_oracle(models, name):
    m = models[name]
    gs, os_ = sb.SanchoSolver(m), oracle_lib.sancho_solver(m)
    x = noisy_input(os_, 0.25, 1)
    Sg, So = gs.self_energies(x), os_.self_energies(x)
    for k, (a, b) in enumerate(zip(Sg, So)):
        if m.order < 3 and k >= 2:
            assert not np.any(a) and not np.any(b)
            continue
        assert np.max(np.abs(b)) > 0
        assert rel(a, b) < 1e-11, (k, rel(a, b))


@pytest.mark.parametrize("name", [n for n, _ in MODELS])
def test_initial_vector_and_residual_match_oracle(models, name):
    m = models[name]
    gs, os_ = sb.SanchoSolver(m), oracle_lib.sancho_solver(m)
    assert gs.n_vec == os_.n_vec == 3 * m.N_sites ** 2 * m.n_omega
    x0g, x0o = gs.initial_vector(-0.3), os_.initial_vector(-0.3)
    assert rel(x0g, x0o) < 1e-12
    x = noisy_input(os_, -0.3, 2)
    (Fg, ag), (Fo, ao) = gs.residual(-0.3, x), os_.residual(-0.3, x)
    assert ag == ao
    scale = np.max(np.abs(Fo + x))
    assert np.max(np.abs(Fg - Fo)) / scale < 1e-11


@pytest.mark.parametrize("name", ["o0", "o1", "o2", "o3", "o3_long", "o2_single_site"])
def test_voltage_sweep_matches_oracle(models, name):
    """The program's voltage loop (continuation on a converged point): same Broyden steps,
    convergence, currents and observables as the oracle."""
    m = models[name]
    gs, os_ = sb.SanchoSolver(m), oracle_lib.sancho_solver(m)
    ok_g = ok_o = False
    for k in range(m.n_volt_steps + 1):
        V = m.V + k * m.delv  # src/sancho.f90's voltage loop
        fresh_g, fresh_o = k == 0 or not ok_g, k == 0 or not ok_o
        rg, ro = gs.solve_scf(V, fresh_g), os_.solve_scf(V, fresh_o)
        ok_g, ok_o = rg["converged"], ro["converged"]
        assert ok_g == ok_o and rg["n_iter"] == ro["n_iter"], (V, rg, ro)
        for key in ("aborted", "runaway", "unphysical"):
            assert rg[key] == ro[key], (V, key)
        # the worst state (check_gf_sanity's report): its spectral weight agrees; the state
        # itself and its occupation agree unless two states tie in spectral weight (the
        # mirror-symmetric chain's end sites do exactly, and rounding picks either)
        assert abs(rg["w_worst"] - ro["w_worst"]) < 1e-9, (V, rg["w_worst"], ro["w_worst"])
        if rg["i_worst"] == ro["i_worst"]:
            assert abs(rg["n_worst"] - ro["n_worst"]) < 1e-9, (V, rg["n_worst"], ro["n_worst"])
        Jg, Jo = gs.current(V), os_.current(V)
        assert abs(Jg - Jo) <= 1e-9 * max(1.0, abs(Jo)), (V, Jg, Jo)
        og, oo = gs.observables(), os_.observables()
        assert rel(og["G_less_t0"], oo["G_less_t0"]) < 1e-9
        assert rel(og["spectral"], oo["spectral"]) < 1e-9


SANCHO_CASES = g.cases(g.GOLDEN_SANCHO)


@pytest.mark.parametrize("case,rc,refs", SANCHO_CASES, ids=[c[0] for c in SANCHO_CASES])
def test_program_reproduces_sancho_regression_case(case, rc, refs, workdir):
    ok, worst, msg, work = g.check_case(sb.PROGRAM, case, rc, refs, os.path.join(workdir, "sancho_b200"),
                                        root=g.GOLDEN_SANCHO)
    assert ok, msg
    if rc == 0:
        assert os.path.exists(os.path.join(work, "spectral_function.dat"))


def test_program_matches_oracle_program_on_a_finer_grid(tmp_path):
    """A case outside the regression suite: the order-3 chain of 6 sites on a grid 2.5x
    finer; every output file of the B200 program equals the oracle program's within the
    reference runner's tolerance."""
    d = case_dir(str(tmp_path), "fine", order=3, N_sites=6, delta=0.004, V=-0.4, Vf=0.4, delv=0.4)
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "cpu")
    shutil.copytree(d, dg)
    shutil.copytree(d, do)
    assert sb.run_program(dg) == 0
    import subprocess
    with open(os.path.join(do, "stdout.txt"), "w") as out:
        assert subprocess.run([oracle_lib.SANCHO_ORACLE_EXE, do], stdout=out, stderr=subprocess.STDOUT,
                              timeout=900).returncode == 0
    for f in ("Volt_Current_3.dat", "populations.dat", "spectral_function.dat"):
        ok, worst, msg = g.compare_files(os.path.join(dg, f), os.path.join(do, f))
        assert ok, msg


def test_site_dependent_u_and_no_continuation_match_oracle(tmp_path):
    """hubbard_file (one U per site, setup_hubbard, SANCHO/src/input_output.f90:106-132) with
    a site at U = 0, and continuation = F (every voltage from the non-interacting start):
    the program's output files equal the oracle program's."""
    d = case_dir(str(tmp_path), "u", order=3, N_sites=5, delta=0.005, hubbard_file="U.dat", continuation="F",
                 V=-0.3, Vf=0.3, delv=0.3)
    with open(os.path.join(d, "U.dat"), "w") as f:
        f.write("0.9\n0.0\n0.6\n1.1\n0.4\n")
    dg, do = str(tmp_path / "gpu"), str(tmp_path / "cpu")
    shutil.copytree(d, dg)
    shutil.copytree(d, do)
    assert sb.run_program(dg) == 0
    import subprocess
    with open(os.path.join(do, "stdout.txt"), "w") as out:
        assert subprocess.run([oracle_lib.SANCHO_ORACLE_EXE, do], stdout=out, stderr=subprocess.STDOUT,
                              timeout=900).returncode == 0
    for f in ("Volt_Current_3.dat", "populations.dat", "spectral_function.dat"):
        ok, worst, msg = g.compare_files(os.path.join(dg, f), os.path.join(do, f))
        assert ok, msg
    m = sb.SanchoModel.load(d)
    assert list(m.U_site) == [0.9, 0.0, 0.6, 1.1, 0.4] and not m.continuation
