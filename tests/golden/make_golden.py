"""Generates tests/golden/pdhg_golden.npz from the reference's own solver.

Run where the reference was compiled into oracle/_ref (make -C oracle ref):

    python tests/golden/make_golden.py

For each known-answer LP, the seeded 1000 x 1500 random LP and four cases of
the 24-period refinery stack it stores what the reference's solve_pdhg
(cpu_backend, default options) returns: status, objective, iteration,
restart and polish counts, and x, y. The tests check the oracle and the
engine against these without needing the reference at run time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from anukulan_b200 import lpgen  # noqa: E402
import lp_cases  # noqa: E402

REFINERY_CASES = (0, 33, 45, 55)


def problems():
    for name, (builder, _, _) in lp_cases.KNOWN.items():
        yield name, lp_cases.standard(builder()), dict(tolerance=1e-8)
    lp, _ = lpgen.random_lp()
    yield "random_1000x1500", lp, dict(tolerance=1e-6)
    stack = lpgen.refinery_stack()
    for k in REFINERY_CASES:
        yield f"refinery_case{k}", stack.case(k), dict(tolerance=1e-6)


def main():
    out = {}
    for name, lp, opts in problems():
        r = oracle.ref_solve(lp, **opts)
        out[f"{name}/status"] = np.int32(r.status)
        out[f"{name}/objective"] = np.float64(r.objective)
        out[f"{name}/iterations"] = np.int32(r.iterations)
        out[f"{name}/restarts"] = np.int32(r.restarts)
        out[f"{name}/polish_attempts"] = np.int32(r.polish_attempts)
        out[f"{name}/x"] = r.x
        out[f"{name}/y"] = r.y
        out[f"{name}/tolerance"] = np.float64(opts["tolerance"])
        print(name, r.status_name, r.iterations, r.objective)
    np.savez_compressed(os.path.join(HERE, "pdhg_golden.npz"), **out)


if __name__ == "__main__":
    main()
