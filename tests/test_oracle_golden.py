"""The oracle pinned to the reference's golden vectors: every case of the reference's
regression suites (tests/cases.txt for QUICHOTTE, SANCHO/tests/cases.txt for SANCHO)
through the oracle programs, compared as the reference's own runner does (1e-6 abs +
1e-5 rel, tests/run_tests.f90:14)."""
import os

import pytest

import golden_runner as g
import oracle_lib

CASES = g.cases()


@pytest.mark.parametrize("case,rc,refs", CASES, ids=[c[0] for c in CASES])
def test_oracle_reproduces_reference_case(case, rc, refs, workdir):
    ok, worst, msg, work = g.check_case(oracle_lib.ORACLE_EXE, case, rc, refs, os.path.join(workdir, "oracle"),
                                        env={"OMP_NUM_THREADS": "4"})
    assert ok, msg


SANCHO_CASES = g.cases(g.GOLDEN_SANCHO)


@pytest.mark.parametrize("case,rc,refs", SANCHO_CASES, ids=[c[0] for c in SANCHO_CASES])
def test_sancho_oracle_reproduces_reference_case(case, rc, refs, workdir):
    ok, worst, msg, work = g.check_case(oracle_lib.SANCHO_ORACLE_EXE, case, rc, refs,
                                        os.path.join(workdir, "sancho_oracle"), env={"OMP_NUM_THREADS": "4"},
                                        root=g.GOLDEN_SANCHO)
    assert ok, msg
