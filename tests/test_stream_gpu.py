"""Streaming case stacks (anu_pdhg_batch_stream): cases admitted from a
source as slots free up, results handed to a sink as cases retire.

- Ten refinery cases streamed through 4 slots end as their single solves do
  (FP64: same status, iterations within two check periods, objectives to
  1e-8 relative, as the rolling stack is held to), each result once.
- A source that reads the sink's results: every retired case may add a child
  (its supply bound halved), as branch and bound adds the children of a
  solved node. All cases come back, children after their parents, and FP32
  results meet the tolerance when the oracle re-evaluates them in FP64.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stack():
    return lpgen.refinery_stack()


def test_stream_equals_single_solves(engine, stack):
    ids = list(range(10))
    solver = engine.CaseStackSolver(stack.base, stack.c[:1], tolerance=1e-6)
    queue = list(ids)
    got = {}

    def source(case):
        if not queue:
            return None
        k = queue.pop(0)
        case.c[:] = stack.c[k]
        case.q[:] = stack.q[k]
        case.lower[:] = stack.lower[k]
        case.upper[:] = stack.upper[k]
        return k

    def sink(k, result):
        assert k not in got
        got[k] = result

    solver.stream(source, sink, slots=4)
    solver.close()
    assert sorted(got) == ids
    for k in ids:
        single = engine.solve_pdhg(stack.case(k), tolerance=1e-6)
        r = got[k]
        assert r.status == single.status == OPTIMAL, k
        assert abs(r.iterations - single.iterations) <= 80, k
        assert abs(r.objective - single.objective) <= 1e-8 * abs(single.objective), k


def test_stream_children_from_results(engine, stack):
    base = stack.base
    solver = engine.CaseStackSolver(base, stack.c[:1], tolerance=1e-6, precision=PRECISION_FP32)
    supply = np.flatnonzero(np.isfinite(base.upper))[:3]
    queue = [(i, None) for i in range(3)]          # (id, parent id)
    parent_of = {}
    order = []
    got = {}
    next_id = [3]

    def source(case):
        if not queue:
            return None
        k, parent = queue.pop(0)
        if parent is not None:
            j = supply[parent % len(supply)]
            case.upper[j] = 0.5 * base.upper[j]
        parent_of[k] = parent
        return k

    def sink(k, result):
        got[k] = result
        order.append(k)
        if k < 3:                                    # roots get one child each
            queue.append((next_id[0], k))
            next_id[0] += 1

    solver.stream(source, sink, slots=2)
    solver.close()
    assert sorted(got) == list(range(6))
    for k, parent in parent_of.items():
        if parent is not None:
            assert order.index(parent) < order.index(k)
    for k, r in got.items():
        case = base
        if parent_of[k] is not None:
            up = base.upper.copy()
            j = supply[parent_of[k] % len(supply)]
            up[j] = 0.5 * base.upper[j]
            case = base.with_vectors(upper=up)
        assert r.status == OPTIMAL, (k, r.message)
        assert oracle.oracle_residual(case, r.x, r.y).converged(1e-6), k


def test_stream_rejects_bad_arguments(engine, stack):
    solver = engine.CaseStackSolver(stack.base, stack.c[:1], tolerance=1e-6)
    with pytest.raises(engine.EngineError):
        solver.stream(lambda case: None, lambda k, r: None, slots=0)

    def bad(case):
        case.lower[0] = 1.0
        case.upper[0] = 0.0
        return 0

    with pytest.raises(engine.EngineError):
        solver.stream(bad, lambda k, r: None, slots=2)
    solver.close()
