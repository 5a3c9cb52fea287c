"""Crossover from the engine's first-order points, on the B200.

- The CLI's `simplex --crossover` (app/anukulan_cli.cpp:574-636) as one
  call, anu_b200::solve_model_crossover, with the PDHG seed on the engine
  through the LinAlgBackend adapter: presolve, a seed at 1e-4, the
  reference's crossover_basis and simplex, postsolve. It ends at the simplex
  optimum (HiGHS, 1e-9) in fewer pivots than the pipeline's cold simplex.
- The case stack's exact stage: the engine bounds every case of the 60-case
  refinery stack at once (FP32, relative KKT 1e-6), its point for the base LP
  goes through crossover_basis and the simplex, and every case is finished by
  the warm dual simplex from that basis (the reference's family --from-first
  step, app/anukulan_cli.cpp:1065-1230). Every case's objective equals the
  reference dual simplex golden to 1e-9; each case whose warm start misses
  is finished from its own engine point instead.
"""
import os

import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import OPTIMAL, PRECISION_FP32
from anukulan_b200.model import to_standard_form
from golden.make_simplex_golden import highs_objective

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not oracle.have_reference_b200(),
                       reason="oracle/_ref adapter build absent"),
]

GOLD = os.path.join(os.path.dirname(__file__), "golden", "simplex_objectives.npz")


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def test_crossover_pipeline_on_engine(engine):
    model, _ = lpgen.refinery_model(24, lpgen.BASE_SEED + 2)
    optimum = highs_objective(to_standard_form(model).lp)[1]
    rc, x, seeded = oracle.ref_pipeline_crossover(model, engine=True, use_presolve=True)
    rc_c, _, cold = oracle.ref_pipeline_crossover(model, engine=True, use_presolve=True,
                                                  crossover_tolerance=0.0)
    assert rc == rc_c == 0
    assert seeded["status"] == cold["status"] == 0
    assert seeded["seeded"] == 1 and seeded["seed_status"] == OPTIMAL
    assert rel(seeded["objective"], optimum) <= 1e-9
    assert seeded["row_violation"] <= 1e-9
    assert seeded["pivots"] < cold["pivots"]


def test_case_stack_finished_exactly(engine):
    stack = lpgen.refinery_stack()
    gold = np.load(GOLD)["refinery/objective"]
    bounds = engine.solve_case_stack(stack, tolerance=1e-6, precision=PRECISION_FP32)
    assert all(r.status == OPTIMAL for r in bounds)
    base = engine.solve_pdhg(stack.base, tolerance=1e-6, precision=PRECISION_FP32)
    assert base.status == OPTIMAL
    fin = oracle.ref_finish_simplex(stack.base, base.x, base.y)
    assert fin["status"] == 0 and fin["seeded"] == 1
    cold, _ = oracle.ref_simplex_basis(stack.base)
    assert fin["pivots"] < cold["pivots"]
    for k in range(stack.num_cases):
        warm, _ = oracle.ref_simplex_basis(stack.case(k), fin["basis"])
        if warm["status"] != 0:
            own = oracle.ref_finish_simplex(stack.case(k), bounds[k].x, bounds[k].y)
            warm = {"status": own["status"], "objective": own["objective"]}
        assert warm["status"] == 0, k
        assert rel(warm["objective"], gold[k]) <= 1e-9, (k, warm["objective"], gold[k])
        # The engine's first-order objective brackets the exact one to the
        # relative gap its KKT tolerance allows (about twice the tolerance).
        assert rel(bounds[k].objective, gold[k]) <= 2e-6, k
