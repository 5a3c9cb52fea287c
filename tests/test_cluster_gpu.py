"""Cluster-resident chunks (options.cluster_chunks): a single LP whose y and
x_bar fit in one CTA's shared memory runs each check period as one launch of
one thread-block cluster, instead of two launches per iteration.

The cluster kernel sums every row in rows_kernel's order and runs the same
step epilogues, so the tests hold it to bit-identical iterates, iteration
and restart counts against cluster_chunks=0, FP32 and FP64:
- the 1000 x 1500 random LP and a refinery case, fixed budgets and whole
  solves with polishing (whose single-case sub-solves take the cluster too);
- an LP with rows of 700 nonzeros (the warp-summed rows);
- an LP with rows longer than 1,024 (not taken: the same kernels run);
- a case stack, whose last FP32 case is handed to the single-LP path.
The FP64 iterates also match the oracle to 1e-10 after fixed budgets.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu

PRECISIONS = [0, PRECISION_FP32]


def same(a, b):
    return (a.status == b.status and a.iterations == b.iterations
            and a.restarts == b.restarts and a.polish_attempts == b.polish_attempts
            and np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y))


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


@pytest.fixture(scope="module")
def refinery():
    return lpgen.refinery_stack()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("budget", [1, 40, 57, 400])
def test_fixed_budget_bit_identical(engine, precision, budget):
    lp, _ = lpgen.random_lp()
    kw = dict(max_iterations=budget, polish_on_exit=0, polish_feasibility=0, precision=precision)
    on = engine.solve_pdhg(lp, cluster_chunks=1, **kw)
    off = engine.solve_pdhg(lp, cluster_chunks=0, **kw)
    assert on.status == ITERATION_LIMIT and on.iterations == budget
    assert same(on, off)
    # One launch per chunk instead of two per iteration.
    if budget >= 40:
        assert on.kernel_launches < off.kernel_launches
    if precision == 0:
        o = oracle.oracle_solve(lp, **kw)
        assert on.restarts == o.restarts
        assert rel_err(on.x, o.x) < 1e-10 and rel_err(on.y, o.y) < 1e-10


@pytest.mark.parametrize("precision", PRECISIONS)
def test_whole_solves_bit_identical(engine, refinery, precision):
    for lp in (lpgen.random_lp()[0], refinery.case(46), refinery.case(16)):
        on = engine.solve_pdhg(lp, tolerance=1e-6, precision=precision, cluster_chunks=1)
        off = engine.solve_pdhg(lp, tolerance=1e-6, precision=precision, cluster_chunks=0)
        assert on.status == OPTIMAL, on.message
        assert same(on, off)
        assert oracle.oracle_residual(lp, on.x, on.y).converged(1e-6)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_warp_rows_bit_identical(engine, precision):
    lp = lpgen.long_row_stack().case(3)
    assert 32 < lp.k.row_lengths().max() <= 1024
    kw = dict(max_iterations=600, polish_on_exit=0, polish_feasibility=0, precision=precision)
    on = engine.solve_pdhg(lp, cluster_chunks=1, **kw)
    off = engine.solve_pdhg(lp, cluster_chunks=0, **kw)
    assert same(on, off)
    assert on.kernel_launches < off.kernel_launches


def test_rows_longer_than_1024_not_taken(engine):
    lp = lpgen.long_row_stack(m=2000, n=3000, long_len=2500).case(0)
    kw = dict(max_iterations=200, polish_on_exit=0, polish_feasibility=0)
    on = engine.solve_pdhg(lp, cluster_chunks=1, **kw)
    off = engine.solve_pdhg(lp, cluster_chunks=0, **kw)
    assert same(on, off)
    assert on.kernel_launches == off.kernel_launches


def test_stack_tail_bit_identical(engine, refinery):
    sub = lpgen.CaseStack(refinery.base, refinery.names[10:20], refinery.c[10:20],
                          refinery.q[10:20], refinery.lower[10:20], refinery.upper[10:20])
    kw = dict(tolerance=1e-6, precision=PRECISION_FP32, split_stacks=0)
    on = engine.solve_case_stack(sub, cluster_chunks=1, **kw)
    off = engine.solve_case_stack(sub, cluster_chunks=0, **kw)
    for k, (a, b) in enumerate(zip(on, off)):
        assert a.status == OPTIMAL, (k, a.message)
        assert same(a, b), k


def test_invalid_option_rejected(engine):
    lp, _ = lpgen.random_lp()
    with pytest.raises(Exception, match="cluster_chunks"):
        engine.solve_pdhg(lp, cluster_chunks=2, max_iterations=10)
