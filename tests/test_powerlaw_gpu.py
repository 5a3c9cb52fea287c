"""The 200,000 x 300,000 power-law LP (2.4M nonzeros, row lengths drawn from
a power law with exponent 2.2 on [3, 5000], 8 nonzeros per column) at full
size, through the C ABI.

- FP64 iterates after a fixed number of iterations match the oracle (the
  restated reference solve_pdhg) to 1e-10 relative, with the same restart
  count. At this size the oracle's serial FP64 iteration takes a few
  seconds per hundred iterations, so the check stops at 200.
- FP32 iterates with FP64 checks and refinement reach relative KKT 1e-4;
  the oracle re-evaluates the returned point in FP64, and the objective is
  compared with the planted optimum c'x0 of the generator.
- Both hold with the rows and columns relabelled for locality
  (locality_order=1).
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def powerlaw():
    return lpgen.power_law_lp()


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def test_powerlaw_shape(powerlaw):
    lp, _ = powerlaw
    lengths = lp.k.row_lengths()
    assert (lp.num_rows, lp.num_cols, lp.k.nnz) == (200_000, 300_000, 2_400_000)
    assert lengths.min() >= 3 and lengths.max() <= 5000


FIXED = dict(max_iterations=200, polish_on_exit=0, polish_feasibility=0)


@pytest.fixture(scope="module")
def oracle_200(powerlaw):
    return oracle.oracle_solve(powerlaw[0], **FIXED)


@pytest.mark.parametrize("locality_order", [0, 1])
def test_powerlaw_fp64_iterates_match_oracle(engine, powerlaw, oracle_200, locality_order):
    """With locality_order the engine runs on relabelled rows and columns;
    every product entry keeps its summation order, so the iterates, mapped
    back, still match the oracle."""
    lp, _ = powerlaw
    r = engine.solve_pdhg(lp, locality_order=locality_order, **FIXED)
    o = oracle_200
    assert r.status == o.status == ITERATION_LIMIT
    assert r.iterations == o.iterations == 200
    assert r.restarts == o.restarts
    assert rel_err(r.x, o.x) < 1e-10
    assert rel_err(r.y, o.y) < 1e-10


def test_powerlaw_fp32_relabelled_reaches_1e4(engine, powerlaw):
    lp, objective = powerlaw
    r = engine.solve_pdhg(lp, tolerance=1e-4, precision=PRECISION_FP32, max_iterations=400_000,
                          locality_order=1)
    assert r.status == OPTIMAL, r.message
    res = oracle.oracle_residual(lp, r.x, r.y)
    assert res.converged(1e-4), res
    assert abs(r.objective - objective) <= 1e-3 * abs(objective)


def test_powerlaw_fp32_refined_reaches_1e4(engine, powerlaw):
    lp, objective = powerlaw
    r = engine.solve_pdhg(lp, tolerance=1e-4, precision=PRECISION_FP32, max_iterations=400_000)
    assert r.status == OPTIMAL, r.message
    res = oracle.oracle_residual(lp, r.x, r.y)
    assert res.converged(1e-4), res
    assert abs(r.objective - objective) <= 1e-3 * abs(objective)
