"""scale_lp on the device (options.scaling_on_device, the default) against
the host sweeps (scaling_on_device = 0).

The device sweeps take the same norms in the same summation order, the same
correctly rounded factors and the same two roundings per nonzero
(src/anukulan/scaling.cpp:32-100, sparse.cpp:120-160), so the scaled matrix
is bit-identical. Everything downstream is then the same computation, so
FP64 solves agree bit for bit: iteration and restart counts, ||K|| and every
entry of x and y. The scaling spreads the result reports agree exactly too.
"""
import numpy as np
import pytest

import lp_cases
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.status == b.status
    assert a.iterations == b.iterations and a.restarts == b.restarts
    assert a.matrix_norm_estimate == b.matrix_norm_estimate
    assert a.spreads == b.spreads
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


@pytest.mark.parametrize("make", [
    lambda: lpgen.random_lp()[0],
    lambda: lpgen.refinery_stack().case(46),
    lambda: lp_cases.standard(lp_cases.boxed_free()),
], ids=["random_1000x1500", "refinery_case_46", "boxed_free"])
def test_device_scaling_solves_bit_identical(engine, make):
    lp = make()
    host = engine.solve_pdhg(lp, tolerance=1e-6, scaling_on_device=0)
    dev = engine.solve_pdhg(lp, tolerance=1e-6, scaling_on_device=1)
    assert dev.status == OPTIMAL
    _same(host, dev)


def test_device_scaling_powerlaw_iterates_bit_identical(engine):
    lp, _ = lpgen.power_law_lp()
    kw = dict(max_iterations=200, polish_on_exit=0, polish_feasibility=0)
    host = engine.solve_pdhg(lp, scaling_on_device=0, **kw)
    dev = engine.solve_pdhg(lp, scaling_on_device=1, **kw)
    assert dev.status == ITERATION_LIMIT
    _same(host, dev)


def test_device_scaling_case_stack_bit_identical(engine):
    stack = lpgen.refinery_stack()
    sel = slice(0, 6)
    args = (stack.base, stack.c[sel], stack.q[sel], stack.lower[sel], stack.upper[sel])
    out = []
    for flag in (0, 1):
        solver = engine.CaseStackSolver(*args, tolerance=1e-6, scaling_on_device=flag)
        out.append(solver.solve())
        solver.close()
    for a, b in zip(*out):
        assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
        assert a.iterations == b.iterations


def test_device_scaling_options_without_sweeps(engine):
    """No sweeps at all, or the 1-norm sweep alone."""
    lp, _ = lpgen.random_lp(300, 450, 8, seed=4)
    for kw in (dict(ruiz_iterations=0, pock_chambolle=0), dict(ruiz_iterations=0),
               dict(pock_chambolle=0)):
        host = engine.solve_pdhg(lp, tolerance=1e-6, scaling_on_device=0, **kw)
        dev = engine.solve_pdhg(lp, tolerance=1e-6, scaling_on_device=1, **kw)
        _same(host, dev)
    r32 = engine.solve_pdhg(lp, tolerance=1e-6, precision=PRECISION_FP32)
    assert r32.status == OPTIMAL
