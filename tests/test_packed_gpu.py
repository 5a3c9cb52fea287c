"""Packed batches of unequal LPs (anu_pdhg_packed_*) through the C ABI.

Each LP of a packed batch runs the same single-LP path as anu_pdhg_solve,
only concurrently with the others, so in FP64 every LP's answer must equal
its own single solve bit for bit. In FP32 with refinement each returned point
is re-evaluated by the oracle in FP64 and must meet relative KKT 1e-6, and
its objective must match the generator's planted optimum c'x0.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    # The construction of the 256-LP workload, smaller: rows log-uniform in
    # [300, 5000], 1.5x as many columns, 8 nonzeros per column.
    return lpgen.packed_batch(count=24, min_rows=300, max_rows=5000, seed=77)


def test_packed_fp64_equals_single_solves(engine, batch):
    lps = [lp for lp, _ in batch[:8]]
    res = engine.solve_packed(lps, workers=4, tolerance=1e-6)
    for lp, r in zip(lps, res):
        s = engine.solve_pdhg(lp, tolerance=1e-6)
        assert r.status == s.status == OPTIMAL
        assert r.iterations == s.iterations
        assert np.array_equal(r.x, s.x) and np.array_equal(r.y, s.y)


def test_packed_fp32_autotuned_reaches_tolerance(engine, batch):
    lps = [lp for lp, _ in batch]
    solver = engine.PackedBatchSolver(lps, tolerance=1e-6, precision=PRECISION_FP32)
    try:
        assert 1 <= solver.workers <= len(lps)
        res = solver.solve()
    finally:
        solver.close()
    for (lp, objective), r in zip(batch, res):
        assert r.status == OPTIMAL, r.message
        assert oracle.oracle_residual(lp, r.x, r.y).converged(1e-6)
        assert abs(r.objective - objective) <= 1e-4 * max(1.0, abs(objective))


def test_packed_rejects_bad_input(engine, batch):
    lp, _ = batch[0]
    with pytest.raises(engine.EngineError):
        engine.solve_packed([lp], workers=-1)


def test_packed_full_batch(engine):
    """The whole 256-LP batch at its real sizes (rows log-uniform in [500,
    50,000]), FP32 with refinement, autotuned worker count. Every LP that
    ends optimal is re-evaluated in FP64 by the engine's evaluate_residual and
    meets relative KKT 1e-6, with its objective at the planted optimum c'x0
    to 1e-5; the rest may only stop at the iteration limit (the reference's
    PDHG needs more than its 200,000 iterations on a few members)."""
    from anukulan_b200.abi import ITERATION_LIMIT
    full = lpgen.packed_batch()
    lps = [lp for lp, _ in full]
    solver = engine.PackedBatchSolver(lps, tolerance=1e-6, precision=PRECISION_FP32)
    try:
        res = solver.solve()
    finally:
        solver.close()
    optimal = 0
    for (lp, objective), r in zip(full, res):
        assert r.status in (OPTIMAL, ITERATION_LIMIT), r.message
        if r.status != OPTIMAL:
            assert r.iterations >= 200_000
            continue
        optimal += 1
        rr = engine.evaluate_residual(lp, r.x, r.y)
        assert rr.converged(1e-6), rr
        assert abs(r.objective - objective) <= 1e-5 * max(1.0, abs(objective))
    assert optimal >= 250
