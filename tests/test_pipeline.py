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
"""
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
