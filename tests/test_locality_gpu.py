"""The single-LP path with rows and columns relabelled for locality
(options.locality_order = 1), against the oracle and the known optima.

The relabelling runs after scaling and keeps every row's nonzeros in their
original order, so each product entry is summed as without it; only the
check reductions sum in another order. The FP64 tolerances are therefore the
ones the unrelabelled engine meets against the oracle (iterates 1e-10
relative after a fixed number of iterations, same restart count); x, y and
warm starts are in the caller's order.
"""
import numpy as np
import pytest

import lp_cases
import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu

FP64_ITERATE_RTOL = 1e-10


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def test_relabelled_iterates_match_oracle_fp64(engine):
    lp, _ = lpgen.random_lp()
    for n_it in (40, 200, 1000):
        kw = dict(max_iterations=n_it, polish_on_exit=0, polish_feasibility=0)
        r = engine.solve_pdhg(lp, locality_order=1, **kw)
        o = oracle.oracle_solve(lp, **kw)
        assert r.status == o.status == ITERATION_LIMIT
        assert r.iterations == o.iterations == n_it
        assert r.restarts == o.restarts
        assert rel_err(r.x, o.x) < FP64_ITERATE_RTOL, n_it
        assert rel_err(r.y, o.y) < FP64_ITERATE_RTOL, n_it


@pytest.mark.parametrize("name", sorted(lp_cases.KNOWN))
def test_relabelled_known_optima(engine, name):
    builder, objective, x = lp_cases.KNOWN[name]
    lp = lp_cases.standard(builder())
    r = engine.solve_pdhg(lp, tolerance=1e-8, locality_order=1)
    o = oracle.oracle_solve(lp, tolerance=1e-8)
    assert r.status == OPTIMAL
    assert abs(r.objective - objective) <= 1e-6 * max(1.0, abs(objective))
    if x is not None:
        np.testing.assert_allclose(r.x, x, atol=1e-5)
    assert abs(r.iterations - o.iterations) <= 40
    r32 = engine.solve_pdhg(lp, tolerance=1e-6, precision=PRECISION_FP32, locality_order=1)
    assert r32.status == OPTIMAL
    assert oracle.oracle_residual(lp, r32.x, r32.y).converged(1e-6)


def test_relabelled_case_with_inequality_rows(engine):
    """A refinery case: equality and inequality rows are relabelled within
    their own blocks, so the dual cone still starts at num_equalities."""
    case = lpgen.refinery_stack().case(32)
    assert 0 < case.num_equalities < case.num_rows
    plain = engine.solve_pdhg(case, tolerance=1e-6)
    scale = max(1.0, abs(plain.objective))
    r64 = engine.solve_pdhg(case, tolerance=1e-6, locality_order=1)
    assert r64.status == OPTIMAL, r64.message
    assert abs(r64.iterations - plain.iterations) <= 40
    assert abs(r64.objective - plain.objective) <= 1e-9 * scale
    r32 = engine.solve_pdhg(case, tolerance=1e-6, precision=PRECISION_FP32, locality_order=1)
    assert r32.status == OPTIMAL, r32.message
    assert abs(r32.objective - plain.objective) <= 2e-6 * scale
    for r in (r64, r32):
        assert oracle.oracle_residual(case, r.x, r.y).converged(1e-6)


def test_relabelled_warm_start_in_caller_order(engine):
    """A warm start given in the caller's order: after a fixed number of
    iterations from it, the FP64 iterates match the oracle's from the same
    start. A start mapped to the wrong entries follows another trajectory
    (a shuffled start moves x by 7e-2 relative after 200 iterations)."""
    lp, _ = lpgen.random_lp(300, 450, 8, seed=4)
    start = oracle.oracle_solve(lp, tolerance=1e-4)
    kw = dict(max_iterations=200, polish_on_exit=0, polish_feasibility=0)
    r = engine.solve_pdhg(lp, locality_order=1, warm_x=start.x, warm_y=start.y, **kw)
    o = oracle.oracle_solve(lp, warm_x=start.x, warm_y=start.y, **kw)
    assert r.status == o.status == ITERATION_LIMIT
    assert r.restarts == o.restarts
    assert rel_err(r.x, o.x) < FP64_ITERATE_RTOL
    assert rel_err(r.y, o.y) < FP64_ITERATE_RTOL


def test_relabelled_deterministic(engine):
    lp, _ = lpgen.random_lp(300, 450, 8, seed=4)
    a = engine.solve_pdhg(lp, locality_order=1)
    b = engine.solve_pdhg(lp, locality_order=1)
    assert a.iterations == b.iterations and a.restarts == b.restarts
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
