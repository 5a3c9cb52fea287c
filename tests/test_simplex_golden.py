"""The objective oracle of the PDHG path: optimal objectives from the
reference's dual simplex (src/anukulan/simplex.hpp:452), stored in
tests/golden/simplex_objectives.npz by tests/golden/make_simplex_golden.py.

These CPU tests pin the fixture: the reference simplex agrees with scipy's
HiGHS, run independently, on every stored LP, the stored LPs are the ones the
generators still make (HiGHS again, live, on a sample), and the random LP's
simplex objective is its planted optimum c'x0. The GPU tests then hold the
engine's objectives to the fixture.
"""
import os

import numpy as np
import pytest

from anukulan_b200 import lpgen

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "simplex_objectives.npz")

# Two simplex codes on the same LP end at the same vertex objective up to
# rounding; 1e-9 relative leaves room for their different pivoting.
SIMPLEX_RTOL = 1e-9


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.fixture(scope="module")
def golden():
    return np.load(FIXTURE)


def test_refinery_simplex_optimal_and_agrees_with_highs(golden):
    status = golden["refinery/status"]
    obj = golden["refinery/objective"]
    highs = golden["refinery/highs_objective"]
    assert status.shape == (60,) and np.all(status == 0)
    for k in range(60):
        assert _rel(obj[k], highs[k]) <= SIMPLEX_RTOL, (k, obj[k], highs[k])


def test_random_lp_simplex_is_planted_optimum(golden):
    assert int(golden["random_1000x1500/status"]) == 0
    planted = float(golden["random_1000x1500/planted_objective"])
    _, live_planted = lpgen.random_lp()
    assert live_planted == pytest.approx(planted, rel=1e-13)
    assert _rel(float(golden["random_1000x1500/objective"]), planted) <= SIMPLEX_RTOL
    assert _rel(float(golden["random_1000x1500/highs_objective"]), planted) <= SIMPLEX_RTOL


@pytest.mark.parametrize("k", [0, 7, 31, 33, 45, 55])
def test_fixture_matches_live_generator(golden, k):
    # HiGHS on the case the generator makes now: a drift of the generator
    # would move the objective away from the stored simplex value.
    from golden.make_simplex_golden import highs_objective
    stack = lpgen.refinery_stack()
    status, obj = highs_objective(stack.case(k))
    assert status == 0
    assert _rel(obj, float(golden["refinery/objective"][k])) <= SIMPLEX_RTOL


def test_reference_pdhg_objectives_near_simplex(golden):
    # The reference's own FP64 PDHG at relative KKT 1e-6 on all 60 cases:
    # optimal, within 2e-6 of the simplex objective (the relative gap is
    # measured against 1 + |c'x| + |q'y|, about twice the objective), and
    # beyond 1e-6 on exactly one case (46).
    simplex = golden["refinery/objective"]
    pdhg = golden["refinery/pdhg_objective"]
    assert np.all(golden["refinery/pdhg_status"] == 0)
    rel = np.abs(pdhg - simplex) / np.maximum(1.0, np.abs(simplex))
    assert float(rel.max()) <= 2e-6
    assert list(np.nonzero(rel > 1e-6)[0]) == [46]
    # The same solver's results in pdhg_golden.npz, bit for bit.
    g = np.load(os.path.join(HERE, "golden", "pdhg_golden.npz"))
    for k in (0, 33, 45, 55):
        assert float(g[f"refinery_case{k}/objective"]) == float(pdhg[k]), k
        assert int(g[f"refinery_case{k}/iterations"]) == int(golden["refinery/pdhg_iterations"][k])


def test_reference_pdhg_golden_within_1e6_of_simplex(golden):
    # The reference's own FP64 PDHG at relative KKT 1e-6 (pdhg_golden.npz)
    # lands within 1e-6 of the simplex objective on the stored cases.
    g = np.load(os.path.join(HERE, "golden", "pdhg_golden.npz"))
    for k in (0, 33, 45, 55):
        pd = float(g[f"refinery_case{k}/objective"])
        assert _rel(pd, float(golden["refinery/objective"][k])) <= 1e-6, k
