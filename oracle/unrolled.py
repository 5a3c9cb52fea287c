"""Test infrastructure: a float64 numpy restatement of the unrolled PDHG
program that anu_pdhg_forward_unrolled runs, and central finite differences of
a loss through it. The unrolled program has no counterpart in the reference
(whose solve_pdhg adapts its restarts); its steps are those of the engine's
own iteration (reflected Halpern PDHG, pdhg.cpp:759-897, backend.cpp:60-111)
with the step sizes held fixed and the Halpern anchor restarted every
`period` steps. Only the tests import this module, as the checker of the
engine's forward pass and of its hand-written adjoint.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import oracle_scale


class ScaledLp:
    """The scaled problem of `lp` (Ruiz + Pock-Chambolle, as solve_pdhg
    scales it), with the diagonal scalings to map vectors in and out."""

    def __init__(self, lp):
        s = oracle_scale(lp)
        self.lp = lp
        self.k = sp.csr_matrix((s["k_value"], lp.k.index, lp.k.start),
                               shape=(lp.num_rows, lp.num_cols))
        self.kt = self.k.T.tocsr()
        self.row_scale = s["row_scale"]
        self.col_scale = s["col_scale"]
        self.lower = s["lower"]
        self.upper = s["upper"]
        self.num_eq = lp.num_equalities

    def scale_c(self, c):
        return np.asarray(c, np.float64) * self.col_scale

    def scale_q(self, q):
        return np.asarray(q, np.float64) * self.row_scale


def forward(slp: ScaledLp, c, q, tau, sigma, iterations, period):
    """x_T and y_T (unscaled) of the unrolled program for objective c and
    right-hand side q (unscaled)."""
    cs = slp.scale_c(c)
    qs = slp.scale_q(q)
    lo, hi = slp.lower, slp.upper
    x = np.zeros_like(cs)
    x = np.where(x < lo, np.where(np.isfinite(lo), lo, 0.0), x)
    x = np.where(x > hi, np.where(np.isfinite(hi), hi, 0.0), x)
    y = np.zeros_like(qs)
    ax = np.zeros_like(x)
    ay = np.zeros_like(y)
    cone = np.arange(len(qs)) >= slp.num_eq
    for t in range(iterations):
        j = t % period
        a = j / (j + 1.0)
        u = x - tau * (cs - slp.kt @ y)
        v = np.clip(u, lo, hi)
        xbar = v + (v - x)
        if j == 0:
            ax = xbar
            xn = xbar
        else:
            xn = a * xbar + (1.0 - a) * ax
        s = y + sigma * (qs - slp.k @ xbar)
        w = np.where(cone, np.maximum(s, 0.0), s)
        yn = w + (w - y)
        if j == 0:
            ay = yn
            y = yn
        else:
            y = a * yn + (1.0 - a) * ay
        x = xn
    return slp.col_scale * x, slp.row_scale * y


def central_differences(slp: ScaledLp, c, q, loss_x, tau, sigma, iterations, period,
                        c_coords=(), q_coords=(), h=1e-4):
    """dL/dc_j and dL/dq_i for L = loss_x . x_T by central differences."""
    def loss(cc, qq):
        x, _ = forward(slp, cc, qq, tau, sigma, iterations, period)
        return float(np.dot(loss_x, x))

    gc, gq = {}, {}
    for j in c_coords:
        e = np.zeros_like(c)
        e[j] = h
        gc[j] = (loss(c + e, q) - loss(c - e, q)) / (2 * h)
    for i in q_coords:
        e = np.zeros_like(q)
        e[i] = h
        gq[i] = (loss(c, q + e) - loss(c, q - e)) / (2 * h)
    return gc, gq


def adjoint(slp: ScaledLp, c, q, loss_x, tau, sigma, iterations, period):
    """dL/dc and dL/dq (unscaled) for L = loss_x . x_T by reverse mode over
    stored iterates: the same derivative the engine's adjoint kernels take,
    written step by step from the forward recurrence."""
    cs = slp.scale_c(c)
    qs = slp.scale_q(q)
    lo, hi = slp.lower, slp.upper
    cone = np.arange(len(qs)) >= slp.num_eq
    x = np.zeros_like(cs)
    x = np.where(x < lo, np.where(np.isfinite(lo), lo, 0.0), x)
    x = np.where(x > hi, np.where(np.isfinite(hi), hi, 0.0), x)
    y = np.zeros_like(qs)
    ax = np.zeros_like(x)
    ay = np.zeros_like(y)
    masks = []
    for t in range(iterations):
        j = t % period
        a = j / (j + 1.0)
        u = x - tau * (cs - slp.kt @ y)
        mu = (u > lo) & (u < hi)
        v = np.clip(u, lo, hi)
        xbar = v + (v - x)
        s = y + sigma * (qs - slp.k @ xbar)
        ms = ~cone | (s > 0)
        w = np.where(cone, np.maximum(s, 0.0), s)
        yn = w + (w - y)
        masks.append((mu, ms))
        if j == 0:
            ax, x = xbar, xbar
            ay, y = yn, yn
        else:
            x = a * xbar + (1.0 - a) * ax
            y = a * yn + (1.0 - a) * ay
    xh = slp.col_scale * np.asarray(loss_x, np.float64)
    yh = np.zeros_like(qs)
    axh = np.zeros_like(xh)
    ayh = np.zeros_like(yh)
    gc = np.zeros_like(cs)
    gq = np.zeros_like(qs)
    for t in range(iterations - 1, -1, -1):
        j = t % period
        a = j / (j + 1.0)
        mu, ms = masks[t]
        if j == 0:
            ny, nx = yh + ayh, xh + axh
            ayh, axh = np.zeros_like(ayh), np.zeros_like(axh)
        else:
            ny, nx = a * yh, a * xh
            ayh = ayh + (1.0 - a) * yh
            axh = axh + (1.0 - a) * xh
        sh = np.where(ms, 2.0 * ny, 0.0)
        gq += sigma * sh
        xbh = -(slp.kt @ (sigma * sh))
        uh = np.where(mu, 2.0 * nx + 2.0 * xbh, 0.0)
        gc -= tau * uh
        xh = -nx - xbh + uh
        yh = -ny + sh + tau * (slp.k @ uh)
    return slp.col_scale * gc, slp.row_scale * gq
