"""The reference's own solver and its own backend tests, unchanged, on the
engine's kernels through the LinAlgBackend adapter (include/
anu_b200_backend.hpp).

oracle/Makefile (target ref_b200) builds anukulan's unmodified sources and
its tests/test_backend.cpp and tests/test_pdhg.cpp with ANUKULAN_WITH_CUDA,
but with src/anukulan/cuda_backend.cu replaced by
anukulan_b200/integration/cuda_backend_b200.cpp, so anukulan::cuda_backend()
and default_backend() are the adapter over libanu_pdhg.so:

* test_backend runs the reference's backend contract on the adapter and its
  CPU-vs-device agreement table (tests/test_backend.cpp:738-893: elementwise
  to 1e-13..1e-14, reductions to 1e-10..1e-12, maxima exactly);
* test_pdhg runs the reference's solve_pdhg known-answer suite
  (tests/test_pdhg.cpp:400-418) with the adapter as its default backend;
* solve_pdhg through the adapter is compared with solve_pdhg on cpu_backend()
  on the same inputs: same status and iteration count, FP64 iterates within
  1e-10 relative after a fixed number of iterations, objectives within 1e-9.
"""
import subprocess

import numpy as np
import pytest

import lp_cases
import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not oracle.have_reference_b200(),
                       reason="oracle/_ref adapter build absent (make -C oracle ref_b200)"),
]

FP64_ITERATE_RTOL = 1e-10
OBJECTIVE_RTOL = 1e-9


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def _run(path):
    p = subprocess.run([path], capture_output=True, text=True, timeout=600)
    return p.returncode, p.stdout + p.stderr


def test_default_backend_is_the_adapter(engine):
    assert oracle.ref_b200_backend_name() == "b200"


def test_reference_backend_contract_on_engine(engine):
    rc, out = _run(oracle.REF_B200_TEST_BACKEND)
    assert rc == 0, out
    assert "contract: b200" in out, out
    assert "skip cuda" not in out, out
    assert "ok   test_backend" in out, out


def test_reference_pdhg_suite_on_engine(engine):
    rc, out = _run(oracle.REF_B200_TEST_PDHG)
    assert rc == 0, out
    assert "ok   test_pdhg" in out, out


def test_reference_solver_iterates_on_engine_match_cpu_backend(engine):
    lp, _ = lpgen.random_lp()
    for n_it in (40, 200):
        kw = dict(max_iterations=n_it, polish_on_exit=0, polish_feasibility=0)
        g = oracle.ref_b200_solve(lp, **kw)
        c = oracle.ref_solve(lp, threads=1, **kw)
        assert g.status == c.status == ITERATION_LIMIT
        assert g.iterations == c.iterations == n_it
        assert g.restarts == c.restarts
        assert rel_err(g.x, c.x) < FP64_ITERATE_RTOL, n_it
        assert rel_err(g.y, c.y) < FP64_ITERATE_RTOL, n_it


@pytest.mark.parametrize("name", sorted(lp_cases.KNOWN))
def test_reference_solver_on_engine_known_optima(engine, name):
    build, objective, x_known = lp_cases.KNOWN[name]
    lp = lp_cases.standard(build())
    g = oracle.ref_b200_solve(lp, tolerance=1e-8)
    c = oracle.ref_solve(lp, threads=1, tolerance=1e-8)
    assert g.status == c.status == OPTIMAL
    assert abs(g.iterations - c.iterations) <= 40
    assert abs(g.objective - objective) <= 1e-6 * max(1.0, abs(objective))
    assert abs(g.objective - c.objective) <= OBJECTIVE_RTOL * max(1.0, abs(c.objective))


def test_reference_solver_on_engine_full_solves(engine):
    lp, planted = lpgen.random_lp()
    for case, known in ((lp, planted), (lpgen.refinery_stack().case(0), None)):
        g = oracle.ref_b200_solve(case, tolerance=1e-6)
        c = oracle.ref_solve(case, threads=1, tolerance=1e-6)
        assert g.status == c.status == OPTIMAL, g.message
        assert abs(g.iterations - c.iterations) <= 40
        assert abs(g.objective - c.objective) <= OBJECTIVE_RTOL * max(1.0, abs(c.objective))
        assert oracle.ref_residual(case, g.x, g.y).converged(1e-6)
        if known is not None:
            assert abs(g.objective - known) <= 1e-5 * abs(known)


def test_adapter_profile_report(engine):
    """set_profiling / profile_report (backend.hpp:213-214), which the CLI's
    --profile prints: with profiling on, the reference's solve_pdhg through
    the adapter leaves a report of the seam operations it ran, the products
    and the two updates among them, whose shares add up to the total; off,
    the report is empty."""
    lp, _ = lpgen.random_lp(300, 450, 8, seed=20261203)
    engine.backend_set_profiling(True)
    try:
        r = oracle.ref_b200_solve(lp, tolerance=1e-6)
        report = engine.backend_profile_report()
    finally:
        engine.backend_set_profiling(False)
    assert r.status == OPTIMAL
    rows = {}
    for line in report.splitlines()[1:]:
        if not line.strip() or line.startswith("total"):
            break
        name, rest = line[:26].strip(), line[26:].split()
        rows[name] = (float(rest[0]), float(rest[1].rstrip("%")), int(rest[2]))
    for op in ("multiply", "primal update", "dual update", "convergence terms"):
        assert op in rows and rows[op][0] > 0.0 and rows[op][2] > 0, (op, report)
    # Two products per iteration at least.
    assert rows["multiply"][2] >= 2 * r.iterations
    assert abs(sum(v[1] for v in rows.values()) - 100.0) < 0.5
    # The matrices solve_pdhg prepared (K and K'), described although the
    # solve has released them.
    assert "matrices prepared while profiling" in report
    assert report.count(" rows ") >= 2
    assert engine.backend_profile_report() == ""
