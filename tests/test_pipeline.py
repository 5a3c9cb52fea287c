"""anu_b200::solve_model_pdhg (include/anu_b200_pipeline.hpp), the
reference's first-order pipeline as one call: presolve -> standard form ->
solve_pdhg -> postsolve (app/anukulan_cli.cpp:1398-1500). On the CPU it runs
with the reference's cpu_backend(), which pins the steps around the PDHG
solve; tests/test_pipeline_gpu.py runs it on the engine.

Tolerances: without presolve the pipeline is to_standard_form + solve_pdhg,
so x equals a plain solve bit for bit. With presolve at relative KKT 1e-8 the
postsolved x meets the original model's rows to 1e-8 relative and its
objective is the HiGHS optimum to 1e-8. At 1e-6 the reduced model's
tolerance does not carry over to the original, and the CLI's check turns the
answer into a numerical error.

The crossover pipeline and the stack's exact stage run the reference's
crossover_basis and simplex; their objectives are held to the simplex
optimum to 1e-9.
"""
import os

import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import NUMERICAL_ERROR, OPTIMAL
from anukulan_b200.model import to_standard_form
from golden.make_simplex_golden import highs_objective

pytestmark = pytest.mark.skipif(not oracle.have_reference_b200(),
                                reason="oracle/_ref adapter build absent")


@pytest.fixture(scope="module")
def refinery():
    model, _ = lpgen.refinery_model(24, lpgen.BASE_SEED + 2)
    lp = to_standard_form(model).lp
    return model, lp, highs_objective(lp)[1]


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def test_pipeline_without_presolve_is_a_plain_solve(refinery):
    model, lp, _ = refinery
    rc, r, x, y, info = oracle.ref_pipeline(model, use_presolve=False, engine=False,
                                            tolerance=1e-8)
    plain = oracle.ref_solve(lp, threads=1, tolerance=1e-8)
    assert rc == 0 and r.status == plain.status == OPTIMAL
    assert r.iterations == plain.iterations
    assert np.array_equal(x, plain.x)
    assert info[2] == 1.0  # no presolve: the dual is the folded PDHG dual


def test_pipeline_with_presolve_meets_the_original_model(refinery):
    model, _, optimum = refinery
    rc, r, x, y, info = oracle.ref_pipeline(model, use_presolve=True, engine=False,
                                            tolerance=1e-8)
    assert rc == 0 and r.status == OPTIMAL, r.message
    assert len(x) == model.constraints.cols and len(y) == model.constraints.rows
    assert info[1] <= 1e-8
    assert rel(r.objective, optimum) <= 1e-8


def test_pipeline_flags_a_reduced_tolerance_the_original_misses(refinery):
    model, _, _ = refinery
    rc, r, x, y, info = oracle.ref_pipeline(model, use_presolve=True, engine=False,
                                            tolerance=1e-6)
    assert rc == 0
    assert r.status == NUMERICAL_ERROR and info[1] > 1e-6
    assert "original" in r.message


def test_crossover_pipeline_reaches_the_simplex_optimum(refinery):
    """The CLI's `simplex --crossover` (app/anukulan_cli.cpp:574-636) as one
    call, anu_b200::solve_model_crossover: a PDHG seed at 1e-4 on the
    presolved model, crossover_basis, the simplex from that basis. It ends at
    the simplex optimum (HiGHS, to 1e-9) in fewer pivots than the same
    pipeline's cold simplex."""
    model, _, optimum = refinery
    rc, x, seeded = oracle.ref_pipeline_crossover(model, engine=False, use_presolve=True)
    rc_c, x_c, cold = oracle.ref_pipeline_crossover(model, engine=False, use_presolve=True,
                                                    crossover_tolerance=0.0)
    assert rc == rc_c == 0
    assert seeded["status"] == cold["status"] == 0
    assert seeded["seeded"] == 1 and seeded["fell_back"] == 0 and cold["seeded"] == 0
    assert seeded["seed_status"] == OPTIMAL and seeded["seed_iterations"] > 0
    assert rel(seeded["objective"], optimum) <= 1e-9
    assert rel(cold["objective"], optimum) <= 1e-9
    assert seeded["row_violation"] <= 1e-9
    assert seeded["pivots"] < cold["pivots"]


def test_stack_finished_exactly_from_a_crossover_basis():
    """The case stack's exact stage: the base LP's first-order point goes
    through crossover_basis and the simplex, and every case is then finished
    by the warm dual simplex from that basis (the reference's family
    --from-first step, app/anukulan_cli.cpp:1065-1230). Here the seed is the
    reference's own PDHG at 1e-6 on cpu_backend; tests/test_crossover_gpu.py
    takes it from the engine. Cases: a cost, a supply, a demand and a
    capacity case; every objective equals the simplex golden to 1e-9."""
    stack = lpgen.refinery_stack()
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "simplex_objectives.npz"))["refinery/objective"]
    seed = oracle.ref_solve(stack.base, tolerance=1e-6)
    base = oracle.ref_finish_simplex(stack.base, seed.x, seed.y)
    assert base["status"] == 0 and base["seeded"] == 1
    cold, _ = oracle.ref_simplex_basis(stack.base)
    assert base["pivots"] < cold["pivots"]
    assert rel(base["objective"], cold["objective"]) <= 1e-9
    for k in (1, 33, 41, 50):
        warm, _ = oracle.ref_simplex_basis(stack.case(k), base["basis"])
        assert warm["status"] == 0
        assert rel(warm["objective"], gold[k]) <= 1e-9, (k, warm["objective"], gold[k])
        assert warm["pivots"] < cold["pivots"]
