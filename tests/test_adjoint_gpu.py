"""The unrolled PDHG program and its hand-written adjoint
(anu_pdhg_unrolled_*) through the C ABI, on the refinery case stack.

Reference points:
- oracle/unrolled.py, a float64 numpy restatement of the program and of its
  reverse mode, itself pinned against central finite differences in
  test_adjoint_oracle.py;
- central finite differences, h = 1e-4, FP64;
- the envelope theorem at the optimum: d(c'x*)/dc = x*, d(c'x*)/dq = y*,
  with (x*, y*) from the oracle's FP64 solve_pdhg at 1e-9.

Tolerances are relative to the largest entry of the vector compared, and
stated at each check.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import PRECISION_FP32, PRECISION_FP64
from oracle import unrolled as U

pytestmark = pytest.mark.gpu
R = 100


@pytest.fixture(scope="module")
def case():
    stack, c_hat = lpgen.adjoint_case()
    return stack, c_hat, U.ScaledLp(stack.base)


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def test_forward_matches_numpy(engine, case):
    stack, _, slp = case
    base = stack.base
    u = engine.UnrolledPdhg(base, iterations=300, checkpoint_every=R, precision=PRECISION_FP64)
    tau, sigma = u.step_sizes()
    x, y = u.forward()
    u.close()
    xn, yn = U.forward(slp, base.c, base.q, tau[0], sigma[0], 300, R)
    assert rel(x[0], xn) < 1e-10 and rel(y[0], yn) < 1e-10


def test_adjoint_matches_numpy_and_finite_differences(engine, case):
    stack, c_hat, slp = case
    base = stack.base
    u = engine.UnrolledPdhg(base, iterations=300, checkpoint_every=R, precision=PRECISION_FP64)
    tau, sigma = u.step_sizes()
    gc, gq = u.backward(c_hat)
    u.close()
    nc, nq = U.adjoint(slp, base.c, base.q, c_hat, tau[0], sigma[0], 300, R)
    assert rel(gc[0], nc) < 1e-9 and rel(gq[0], nq) < 1e-9
    # Central differences, h = 1e-4, on the largest gradient entries (q: rows
    # with a nonzero right-hand side; see test_adjoint_oracle.py on kinks).
    jc = np.argsort(-np.abs(gc[0]))[:6]
    iq = [i for i in np.argsort(-np.abs(gq[0])) if base.q[i] != 0][:6]
    fc, fq = U.central_differences(slp, base.c, base.q, c_hat, tau[0], sigma[0], 300, R,
                                   jc, iq, h=1e-4)
    for j in jc:
        assert abs(gc[0][j] - fc[j]) <= 1e-6 * np.max(np.abs(gc[0])), j
    for i in iq:
        assert abs(gq[0][i] - fq[i]) <= 1e-6 * np.max(np.abs(gq[0])), i


def test_adjoint_2000_iterations_fp64_and_fp32(engine, case):
    # The workload's length: 2,000 iterations, checkpoints every 100.
    stack, c_hat, slp = case
    base = stack.base
    u64 = engine.UnrolledPdhg(base, iterations=2000, checkpoint_every=R, precision=PRECISION_FP64)
    tau, sigma = u64.step_sizes()
    g64c, g64q = u64.backward(c_hat)
    u64.close()
    nc, nq = U.adjoint(slp, base.c, base.q, c_hat, tau[0], sigma[0], 2000, R)
    assert rel(g64c[0], nc) < 1e-8 and rel(g64q[0], nq) < 1e-8
    u32 = engine.UnrolledPdhg(base, iterations=2000, checkpoint_every=R, precision=PRECISION_FP32)
    g32c, g32q = u32.backward(c_hat)
    u32.close()
    # FP32 iterates and adjoint state, FP64 accumulation. Over 2,000 steps
    # the FP32 trajectory drifts from the FP64 one by rounding (measured
    # 1.2e-3 relative, L2, in dL/dc); 5e-3 relative (L2).
    assert np.linalg.norm(g32c - g64c) <= 5e-3 * np.linalg.norm(g64c)
    assert np.linalg.norm(g32q - g64q) <= 5e-3 * np.linalg.norm(g64q)


def test_batched_cases_equal_single_cases(engine, case):
    stack, c_hat, _ = case
    ratio = c_hat / np.where(stack.base.c != 0, stack.base.c, 1.0)
    ks = [0, 17, 40, 55]
    c = stack.c[ks]
    loss = c * ratio
    ub = engine.UnrolledPdhg(stack.base, c, stack.q[ks], stack.lower[ks], stack.upper[ks],
                             iterations=400, checkpoint_every=R, precision=PRECISION_FP64)
    xb, _ = ub.forward()
    gcb, gqb = ub.backward(loss)
    ub.close()
    for i, k in enumerate(ks):
        us = engine.UnrolledPdhg(stack.case(k), iterations=400, checkpoint_every=R,
                                 precision=PRECISION_FP64)
        xs, _ = us.forward()
        gcs, gqs = us.backward(loss[i])
        us.close()
        assert rel(xb[i], xs[0]) < 1e-10
        assert rel(gcb[i], gcs[0]) < 1e-9 and rel(gqb[i], gqs[0]) < 1e-9


def test_envelope_theorem(engine, case):
    # L = c'x_T: dL/dc = x_T + (dx_T/dc)'c -> x*, dL/dq -> y*. 8,000 steps
    # bring x_T within 2e-4 of x*. The 288 rows with a zero right-hand side
    # are degenerate (the optimal value has a kink there and y* is not
    # unique on them), so the dual check covers the other 2,472 rows.
    stack, _, _ = case
    base = stack.base
    star = oracle.oracle_solve(base, tolerance=1e-9)
    u = engine.UnrolledPdhg(base, iterations=8000, checkpoint_every=R, precision=PRECISION_FP64)
    x, _ = u.forward()
    gc, gq = u.backward(base.c)
    u.close()
    dc = x[0] + gc[0]
    assert np.linalg.norm(dc - star.x) <= 2e-2 * np.linalg.norm(star.x)
    nz = base.q != 0
    assert np.linalg.norm(gq[0][nz] - star.y[nz]) <= 2.5e-2 * np.linalg.norm(star.y[nz])


def test_unrolled_rejects_bad_arguments(engine, case):
    stack, _, _ = case
    with pytest.raises(engine.EngineError):
        engine.UnrolledPdhg(stack.base, iterations=0)
    with pytest.raises(engine.EngineError):
        engine.UnrolledPdhg(stack.base, checkpoint_every=0)
