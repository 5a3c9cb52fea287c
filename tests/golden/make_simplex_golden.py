"""Generates tests/golden/simplex_objectives.npz: optimal objectives from the
reference's dual simplex, the objective oracle of the PDHG path.

Run where the reference was compiled into oracle/_ref (make -C oracle ref):

    python tests/golden/make_simplex_golden.py

It solves, with the reference's solve_lp (dual simplex,
src/anukulan/simplex.hpp:452), every case of the 60-case 24-period refinery
stack and the seeded 1000 x 1500 random LP, and stores per LP the simplex
status, objective and iteration count. The same LPs are solved again by
scipy's bundled HiGHS (an independent simplex/IPM) and its objectives are
stored beside them as a cross-check; the random LP also stores its planted
optimum c'x0. For the refinery cases it also stores the objective, status and
iteration count of the reference's own FP64 PDHG (solve_pdhg, cpu_backend,
default options) at relative KKT 1e-6, which is how far from the simplex
objective that tolerance lets PDHG land. The tests check the engine's
objectives against these without the reference at run time.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from anukulan_b200 import lpgen  # noqa: E402


def highs_objective(lp):
    """Optimal objective of a StandardLp (equality rows first, the rest
    K x >= q) by scipy's HiGHS, in the model's sense."""
    import scipy.sparse as sp
    from scipy.optimize import linprog
    k = lp.k
    a = sp.csr_matrix((k.value, k.index, k.start), shape=(k.rows, k.cols))
    me = lp.num_equalities
    bounds = np.stack([np.where(np.isinf(lp.lower), -np.inf, lp.lower),
                       np.where(np.isinf(lp.upper), np.inf, lp.upper)], axis=1)
    kw = {}
    if me > 0:
        kw.update(A_eq=a[:me], b_eq=lp.q[:me])
    if me < k.rows:
        kw.update(A_ub=-a[me:], b_ub=-lp.q[me:])
    r = linprog(lp.c, bounds=bounds, method="highs", **kw)
    if r.status != 0:
        return r.status, float("nan")
    return 0, lp.objective_scale * float(r.fun) + lp.objective_offset


def main():
    out = {}
    stack = lpgen.refinery_stack()
    status, obj, its, hobj, pobj, pst, pits = [], [], [], [], [], [], []
    t0 = time.perf_counter()
    for k in range(stack.num_cases):
        lp = stack.case(k)
        st, o, it, _, _ = oracle.ref_simplex(lp)
        hs, ho = highs_objective(lp)
        pd = oracle.ref_solve(lp, tolerance=1e-6)
        pobj.append(pd.objective)
        pst.append(pd.status)
        pits.append(pd.iterations)
        status.append(st)
        obj.append(o)
        its.append(it)
        hobj.append(ho)
        print(f"refinery case {k:2d} {stack.names[k]:28s} simplex {st} {o:.12g} ({it} it)"
              f"  highs {hs} {ho:.12g}  pdhg {pd.objective:.12g} ({pd.iterations} it)")
    out["refinery/status"] = np.array(status, np.int32)
    out["refinery/objective"] = np.array(obj)
    out["refinery/iterations"] = np.array(its, np.int32)
    out["refinery/highs_objective"] = np.array(hobj)
    out["refinery/pdhg_objective"] = np.array(pobj)
    out["refinery/pdhg_status"] = np.array(pst, np.int32)
    out["refinery/pdhg_iterations"] = np.array(pits, np.int32)
    print(f"refinery stack: {time.perf_counter() - t0:.1f} s")

    lp, planted = lpgen.random_lp()
    t0 = time.perf_counter()
    st, o, it, _, _ = oracle.ref_simplex(lp, time_limit=1200.0)
    hs, ho = highs_objective(lp)
    out["random_1000x1500/status"] = np.int32(st)
    out["random_1000x1500/objective"] = np.float64(o)
    out["random_1000x1500/iterations"] = np.int32(it)
    out["random_1000x1500/highs_objective"] = np.float64(ho)
    out["random_1000x1500/planted_objective"] = np.float64(planted)
    print(f"random 1000x1500: simplex {st} {o:.12g} ({it} it, {time.perf_counter() - t0:.1f} s)"
          f"  highs {ho:.12g}  planted {planted:.12g}")
    np.savez_compressed(os.path.join(HERE, "simplex_objectives.npz"), **out)


if __name__ == "__main__":
    main()
