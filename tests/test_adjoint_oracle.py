"""The numpy restatement of the unrolled PDHG program and of its reverse
mode (oracle/unrolled.py), checked on the CPU against central finite
differences, h = 1e-4, in float64, on the refinery base case.

The program is piecewise linear. Its derivative is exact away from the
kinks of the projections. 192 inequality rows of this LP have a zero
right-hand side, and on those rows the cone projection starts exactly at its
kink: y0 = 0 and K x_bar vanishes there. Central differences in those q
coordinates average the two one-sided slopes, while reverse mode takes the
slope with the projection inactive. The q coordinates checked are therefore
rows with a nonzero right-hand side. The c coordinates are the largest
entries of the gradient.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from oracle import unrolled as U

T, R = 300, 100


@pytest.fixture(scope="module")
def setup():
    stack, c_hat = lpgen.adjoint_case()
    base = stack.base
    slp = U.ScaledLp(base)
    eta = 0.9 / oracle.oracle_matrix_norm(base, scaled=True)
    omega = np.linalg.norm(slp.scale_c(base.c)) / np.linalg.norm(slp.scale_q(base.q))
    return base, slp, c_hat, eta / omega, eta * omega


def test_reverse_mode_matches_central_differences(setup):
    base, slp, c_hat, tau, sigma = setup
    gc, gq = U.adjoint(slp, base.c, base.q, c_hat, tau, sigma, T, R)
    jc = np.argsort(-np.abs(gc))[:6]
    iq = [i for i in np.argsort(-np.abs(gq)) if base.q[i] != 0][:6]
    fc, fq = U.central_differences(slp, base.c, base.q, c_hat, tau, sigma, T, R, jc, iq, h=1e-4)
    for j in jc:
        assert abs(gc[j] - fc[j]) <= 1e-6 * np.max(np.abs(gc)), j
    for i in iq:
        assert abs(gq[i] - fq[i]) <= 1e-6 * np.max(np.abs(gq)), i


def test_reverse_mode_matches_directional_difference_off_the_kinks(setup):
    # With q moved off the kinks, a random direction in q agrees too.
    base, slp, c_hat, tau, sigma = setup
    rng = np.random.default_rng(5)
    q = base.q + 1e-3 * rng.uniform(0.5, 1.0, base.num_rows)
    d = rng.standard_normal(base.num_rows)
    _, gq = U.adjoint(slp, base.c, q, c_hat, tau, sigma, 20, R)
    h = 1e-4
    lp = float(c_hat @ U.forward(slp, base.c, q + h * d, tau, sigma, 20, R)[0])
    lm = float(c_hat @ U.forward(slp, base.c, q - h * d, tau, sigma, 20, R)[0])
    assert abs(float(gq @ d) - (lp - lm) / (2 * h)) <= 1e-6 * abs(float(gq @ d))
