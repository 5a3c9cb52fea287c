"""Branch-and-bound node relaxations as one case stack
(pdhg.solve_node_relaxations), against the engine's single solves, the
reference's own solve_pdhg per node (oracle/_ref, cpu_backend) and HiGHS.

The nodes are children of the refinery base case: the three columns whose
root values are most fractional (among values >= 0.5), each branched down
(upper = floor) and up (lower = ceil). Two of the up-branches are infeasible
by HiGHS; the reference's PDHG neither proves that nor converges there, so
every node is capped at 40,000 iterations.

Tolerances: a certified bound (PDHG optimal and dual_residual_inf <= 1e-7 of
the dual objective, branch_and_bound.cpp:560-565) equals the single solve's
and the reference's to 1e-8 relative in FP64. By weak duality it lies below
the node's optimum, up to what the admitted dual infeasibility allows (1e-6
relative here), and within 1e-5 of it. An infeasible node is never certified.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import PRECISION_FP32
from anukulan_b200.pdhg import NodeRelaxation
from golden.make_simplex_golden import highs_objective

pytestmark = pytest.mark.gpu

NODE_ITERATIONS = 40_000
KW = dict(tolerance=1e-6, max_iterations=NODE_ITERATIONS)


def branch(lp, x, count):
    frac = np.abs(x - np.round(x))
    frac[x < 0.5] = 0.0
    lower, upper = [], []
    for j in np.argsort(-frac, kind="stable")[:count]:
        for down in (True, False):
            lo, up = lp.lower.copy(), lp.upper.copy()
            if down:
                up[j] = np.floor(x[j])
            else:
                lo[j] = np.ceil(x[j])
            lower.append(lo)
            upper.append(up)
    return np.array(lower), np.array(upper)


@pytest.fixture(scope="module")
def nodes():
    lp = lpgen.refinery_stack().case(0)
    root = oracle.ref_solve(lp, tolerance=1e-8)
    lower, upper = branch(lp, root.x, 3)
    lps = [lp.with_vectors(lower=lower[k], upper=upper[k]) for k in range(len(lower))]
    highs = [highs_objective(node) for node in lps]
    return lp, lower, upper, lps, highs


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def test_node_stack_equals_single_solves(engine, nodes):
    lp, lower, upper, lps, _ = nodes
    stack = engine.solve_node_relaxations(lp, lower, upper, **KW)
    assert len(stack) == len(lps) == 6
    for k, nd in enumerate(stack):
        single = NodeRelaxation(engine.solve_pdhg(lps[k], **KW))
        assert nd.result.status == single.result.status, k
        assert abs(nd.result.iterations - single.result.iterations) <= 40, k
        assert nd.optimal == single.optimal, k
        if nd.optimal:
            assert rel(nd.bound, single.bound) <= 1e-8, k


def test_node_bounds_match_reference_and_highs(engine, nodes):
    lp, lower, upper, lps, highs = nodes
    stack = engine.solve_node_relaxations(lp, lower, upper, **KW)
    assert sum(nd.optimal for nd in stack) >= 3
    for k, nd in enumerate(stack):
        ref = NodeRelaxation(oracle.ref_solve(lps[k], threads=1, **KW))
        assert nd.result.status == ref.result.status, k
        assert nd.optimal == ref.optimal, k
        status, optimum = highs[k]
        if status != 0:
            assert not nd.optimal, k
        if nd.optimal:
            assert status == 0, k
            assert rel(nd.bound, ref.bound) <= 1e-8, k
            assert nd.bound <= optimum + 1e-6 * max(1.0, abs(optimum)), k
            assert rel(nd.bound, optimum) <= 1e-5, k


def test_node_bounds_fp32(engine, nodes):
    lp, lower, upper, _, highs = nodes
    stack = engine.solve_node_relaxations(lp, lower, upper, precision=PRECISION_FP32, **KW)
    for k, nd in enumerate(stack):
        status, optimum = highs[k]
        if status != 0:
            assert not nd.optimal, k
        if nd.optimal:
            assert rel(nd.bound, optimum) <= 1e-5, k
