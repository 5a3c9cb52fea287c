"""Pins the oracle (oracle/pdhg_oracle.c, the C restatement of the reference
PDHG path) before anything is checked against it:

* against the known optima the reference's own tests hold
  (tests/test_pdhg.cpp:112-470 in anukulan);
* against the golden fixtures generated from the reference's own solver
  (tests/golden/make_golden.py) - bit-exact;
* against the reference compiled from its sources (oracle/_ref), live,
  across option configurations - bit-exact (skipped where it was not built).
"""
import os

import numpy as np
import pytest

import lp_cases
import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRIMAL_INFEASIBLE

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "pdhg_golden.npz")

needs_ref = pytest.mark.skipif(not oracle.have_reference(),
                               reason="oracle/_ref/libanuref.so not built here")


@pytest.mark.parametrize("name", sorted(lp_cases.KNOWN))
def test_oracle_known_optima(name):
    builder, objective, x = lp_cases.KNOWN[name]
    r = oracle.oracle_solve(lp_cases.standard(builder()), tolerance=1e-8)
    assert r.status == OPTIMAL
    assert abs(r.objective - objective) <= 1e-6 * max(1.0, abs(objective))
    if x is not None:
        np.testing.assert_allclose(r.x, x, atol=1e-5)


def test_oracle_matrix_norm_known():
    lp = lp_cases.standard(lp_cases.norm_4())
    assert abs(oracle.oracle_matrix_norm(lp, 500, 1e-12) - 4.0) <= 1e-6


def test_oracle_empty_matrix():
    r = oracle.oracle_solve(lp_cases.standard(lp_cases.empty_rows()), tolerance=1e-8)
    np.testing.assert_allclose(r.x, [0.0, 5.0], atol=1e-6)
    assert abs(r.objective + 5.0) <= 1e-6


def test_oracle_iteration_limit_exact():
    r = oracle.oracle_solve(lp_cases.standard(lp_cases.wyndor()), tolerance=1e-14,
                            max_iterations=80, termination_check_frequency=40)
    assert r.status == ITERATION_LIMIT
    assert r.iterations == 80


def test_oracle_detects_infeasibility():
    r = oracle.oracle_solve(lp_cases.standard(lp_cases.infeasible()), tolerance=1e-8)
    assert r.status == PRIMAL_INFEASIBLE


def test_oracle_deterministic():
    lp = lp_cases.standard(lp_cases.wyndor())
    a = oracle.oracle_solve(lp, tolerance=1e-8)
    b = oracle.oracle_solve(lp, tolerance=1e-8)
    assert a.iterations == b.iterations and a.restarts == b.restarts
    assert np.array_equal(a.x, b.x)


def _golden_problems():
    for name, (builder, _, _) in lp_cases.KNOWN.items():
        yield name, lambda b=builder: lp_cases.standard(b())
    yield "random_1000x1500", lambda: lpgen.random_lp()[0]
    for k in (0, 33, 45, 55):
        yield f"refinery_case{k}", lambda k=k: lpgen.refinery_stack().case(k)


@pytest.mark.parametrize("name,make", list(_golden_problems()), ids=lambda v: v if isinstance(v, str) else "")
def test_oracle_matches_golden_bit_exact(name, make):
    g = np.load(GOLDEN)
    r = oracle.oracle_solve(make(), tolerance=float(g[f"{name}/tolerance"]))
    assert r.status == int(g[f"{name}/status"])
    assert r.iterations == int(g[f"{name}/iterations"])
    assert r.restarts == int(g[f"{name}/restarts"])
    assert r.polish_attempts == int(g[f"{name}/polish_attempts"])
    assert r.objective == float(g[f"{name}/objective"])
    assert np.array_equal(r.x, g[f"{name}/x"])
    assert np.array_equal(r.y, g[f"{name}/y"])


OPTION_SETS = [
    dict(),
    dict(tolerance=1e-8),
    dict(halpern=0),
    dict(restart_on_fixed_point=0),
    dict(pid_primal_weight=0),
    dict(primal_weight_updates=0),
    dict(restarts=0, max_iterations=20000),
    dict(reflection=0.0),
    dict(ruiz_iterations=0, pock_chambolle=0),
    dict(tolerance=1e-8, gap_tolerance=1e-2),
    dict(max_iterations=300),
    dict(reuse_products=0),
    dict(constant_step_size=0, max_iterations=3000),
    dict(halpern_restart=1, max_iterations=3000),
    dict(polish_feasibility=0),
    dict(absolute_tolerance=1e-6),
    dict(require_inf_norm_termination=0),
]


@needs_ref
@pytest.mark.parametrize("opts", OPTION_SETS, ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()) or "defaults")
def test_oracle_equals_reference_across_options(opts):
    lp, _ = lpgen.random_lp(300, 450, 8, seed=11)
    a = oracle.oracle_solve(lp, **opts)
    b = oracle.ref_solve(lp, **opts)
    assert (a.status, a.iterations, a.restarts, a.polish_attempts, a.polish_iterations) == \
        (b.status, b.iterations, b.restarts, b.polish_attempts, b.polish_iterations)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    assert a.objective == b.objective
    assert a.final_primal_weight == b.final_primal_weight
    assert a.final_step_size == b.final_step_size


@needs_ref
@pytest.mark.parametrize("name", sorted(lp_cases.KNOWN) + ["infeasible", "empty_rows"])
def test_oracle_equals_reference_known(name):
    builder = getattr(lp_cases, name)
    lp = lp_cases.standard(builder())
    for opts in (dict(tolerance=1e-8), dict(tolerance=1e-8, warm_x=None)):
        opts = {k: v for k, v in opts.items() if v is not None}
        a = oracle.oracle_solve(lp, **opts)
        b = oracle.ref_solve(lp, **opts)
        assert (a.status, a.iterations, a.restarts) == (b.status, b.iterations, b.restarts)
        assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


@needs_ref
def test_oracle_warm_start_equals_reference():
    lp = lp_cases.standard(lp_cases.wyndor())
    cold = oracle.ref_solve(lp, tolerance=1e-8)
    kw = dict(tolerance=1e-8, ruiz_iterations=0, pock_chambolle=0)
    a = oracle.oracle_solve(lp, warm_x=cold.x, warm_y=cold.y, **kw)
    b = oracle.ref_solve(lp, warm_x=cold.x, warm_y=cold.y, **kw)
    assert a.iterations == b.iterations < cold.iterations
    assert np.array_equal(a.x, b.x)


@needs_ref
def test_oracle_scaling_and_norm_equal_reference():
    lp, _ = lpgen.random_lp(300, 450, 8, seed=5)
    a = oracle.oracle_scale(lp)
    b = oracle.ref_scale(lp)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert oracle.oracle_matrix_norm(lp, scaled=True) == oracle.ref_matrix_norm(lp, scaled=True)


@needs_ref
def test_oracle_residual_equals_reference():
    lp, _ = lpgen.random_lp(300, 450, 8, seed=5)
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 10, lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    a = oracle.oracle_residual(lp, x, y)
    b = oracle.ref_residual(lp, x, y)
    assert a == b
