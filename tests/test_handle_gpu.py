"""anu_pdhg_set_case: one handle, one prepared matrix, many LPs.

A handle keeps its scaled matrix, product schedules and ||K~|| when
anu_pdhg_set_case swaps in another objective, right-hand side and bounds
(the reference's backends keep a prepared matrix per SparseMatrix::id(),
src/anukulan/cuda_backend.cu:561-588). Scaling factors depend on the matrix
alone, so each run must be the run a fresh anu_pdhg_solve of that LP makes:
in FP64 the same status, iteration and restart counts and bit-identical x
and y. Also with the locality relabelling, where the handle maps the new
vectors into its order, and with vectors left NULL (kept).
"""
import numpy as np
import pytest

from anukulan_b200 import lpgen
from anukulan_b200.abi import PRECISION_FP64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("locality", [0, 1])
def test_set_case_runs_equal_fresh_solves(engine, locality):
    st = lpgen.refinery_stack()
    opts = dict(tolerance=1e-6, precision=PRECISION_FP64, locality_order=locality)
    h = engine.PdhgHandle(st.base, **opts)
    try:
        for k in (3, 35, 44, 52):
            h.set_case(st.c[k], st.q[k], st.lower[k], st.upper[k])
            a = h.run()
            b = engine.solve_pdhg(st.case(k), **opts)
            assert a.status == b.status
            assert a.iterations == b.iterations and a.restarts == b.restarts
            assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
            assert a.objective == b.objective
        # NULL keeps a vector: only the objective of case 7 moves.
        h.set_case(st.c[7])
        a = h.run()
        case = st.case(52).with_vectors(c=st.c[7])
        b = engine.solve_pdhg(case, **opts)
        assert a.iterations == b.iterations and np.array_equal(a.x, b.x)
    finally:
        h.close()


def test_set_case_rejects_bad_vectors(engine):
    st = lpgen.refinery_stack()
    h = engine.PdhgHandle(st.base, tolerance=1e-6)
    try:
        lo = st.lower[0].copy()
        lo[0] = st.upper[0][0] + 1.0
        with pytest.raises(engine.EngineError):
            h.set_case(lower=lo)
        with pytest.raises(ValueError):
            h.set_case(c=np.zeros(3))
    finally:
        h.close()
