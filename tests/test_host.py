"""Host-side logic: the standard form's integer maps, the workload
generators' invariants, the ABI structs and defaults, and that the engine
library loads and exports every symbol its header declares."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import lp_cases
import oracle
from anukulan_b200 import abi, lpgen
from anukulan_b200.model import Csr, Model, to_standard_form

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not oracle.have_reference(),
                               reason="oracle/_ref/libanuref.so not built here")


def _mixed_model(seed=0):
    """Equality, >=, <=, ranged and free rows; free, boxed and one-sided columns."""
    rng = np.random.default_rng(seed)
    m, n = 40, 30
    r, c, v = [], [], []
    for i in range(m):
        for j in rng.choice(n, size=rng.integers(0, 6), replace=False):
            r.append(i)
            c.append(int(j))
            v.append(float(rng.standard_normal()))
    a = Csr.from_triplets(m, n, r, c, v)
    kinds = rng.integers(0, 5, m)
    lo = np.where(kinds == 0, 1.0, np.where(kinds == 1, -2.0, np.where(kinds == 3, -1.0, -np.inf)))
    hi = np.where(kinds == 0, 1.0, np.where(kinds == 2, 3.0, np.where(kinds == 3, 4.0, np.inf)))
    lo[kinds == 4] = -np.inf
    hi[kinds == 4] = np.inf
    clo = np.where(rng.random(n) < 0.2, -np.inf, 0.0)
    chi = np.where(rng.random(n) < 0.5, np.inf, 5.0)
    return Model(a, rng.standard_normal(n), lo, hi, clo, chi, bool(seed % 2), 1.5)


@needs_ref
@pytest.mark.parametrize("seed", range(4))
def test_standard_form_bit_exact_with_reference(seed):
    model = _mixed_model(seed)
    mine = to_standard_form(model)
    ref = oracle.ref_to_standard_form(model)
    assert mine.ok and ref is not None
    lp = mine.lp
    assert lp.num_equalities == ref.num_equalities
    assert np.array_equal(lp.k.start, ref.k.start)
    assert np.array_equal(lp.k.index, ref.k.index)
    assert np.array_equal(lp.k.value, ref.k.value)
    assert np.array_equal(lp.row_origin_row, ref.row_origin_row)
    assert np.array_equal(lp.row_origin_sign, ref.row_origin_sign)
    assert np.array_equal(lp.c, ref.c) and np.array_equal(lp.q, ref.q)
    assert (lp.objective_scale, lp.objective_offset) == (ref.objective_scale, ref.objective_offset)


def test_standard_form_layout():
    lp = lp_cases.standard(lp_cases.range_row())
    # a ranged row becomes a'x >= lo and -a'x >= -hi
    assert lp.num_rows == 2 and lp.num_equalities == 0
    assert list(lp.q) == [5.0, -8.0]
    assert list(lp.row_origin_sign) == [1.0, -1.0]
    w = lp_cases.standard(lp_cases.wyndor())
    assert w.objective_scale == -1.0 and list(w.c) == [-3.0, -5.0]


def test_csr_transpose_roundtrip():
    model = _mixed_model(1)
    a = model.constraints
    t = a.transpose()
    tt = t.transpose()
    assert np.array_equal(tt.start, a.start) and np.array_equal(tt.index, a.index)
    assert np.array_equal(tt.value, a.value)


def test_random_lp_known_optimum():
    lp, obj = lpgen.random_lp(200, 300, 8, seed=2)
    assert lp.k.nnz == 300 * 8
    assert np.all(np.diff(lp.k.transpose().start) == 8)
    # c'x0 = b'y0 at the planted optimum
    rng_lp, obj2 = lpgen.random_lp(200, 300, 8, seed=2)
    assert obj == obj2


def test_power_law_lengths():
    rng = np.random.default_rng(0)
    L = lpgen.power_law_row_lengths(20000, 20000 * 12, rng)
    assert L.sum() == 20000 * 12
    assert L.min() >= 3 and L.max() <= 5000


@pytest.mark.slow
def test_power_law_lp_structure():
    lp, _ = lpgen.power_law_lp(20000, 30000, 8, seed=7)
    lengths = lp.k.row_lengths()
    assert lp.k.nnz == 240000
    assert lengths.min() >= 3 and lengths.max() <= 5000
    t = lp.k.transpose()
    assert np.all(np.diff(t.start) == 8)  # distinct rows per column survived


def test_refinery_stack_shape():
    st = lpgen.refinery_stack()
    assert st.num_cases == 60
    assert st.base.num_rows == 2760 and st.base.num_cols == 3840
    # every case differs from the base in exactly one kind of data
    for k in range(60):
        diffs = sum([not np.array_equal(st.c[k], st.base.c), not np.array_equal(st.q[k], st.base.q),
                     not np.array_equal(st.upper[k], st.base.upper)])
        assert diffs == 1
    # buying nothing is feasible: x = 0 satisfies every row
    kx = st.base.k.multiply(np.zeros(st.base.num_cols))
    eq = st.base.num_equalities
    assert np.all(kx[:eq] == st.base.q[:eq])
    assert np.all(kx[eq:] >= st.base.q[eq:])


def test_python_defaults_match_c_abi_defaults():
    from anukulan_b200 import pdhg
    o = pdhg.default_options()
    d = abi.options_dict(o)
    for k, v in abi.DEFAULTS.items():
        assert d[k] == v, k


@needs_ref
def test_defaults_match_reference_pdhg_options():
    ref = abi.options_dict(oracle.ref_default_options())
    mine = abi.options_dict(abi.make_options())
    for k, v in ref.items():
        if k in ("precision", "refinement", "device", "use_graphs", "profile", "split_stacks",
                 "persistent_chunks", "locality_order", "scaling_on_device", "tile_threads",
                 "cluster_chunks"):
            continue
        assert mine[k] == v, k


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "anu_pdhg.h")).read()
    return sorted(set(re.findall(r"\b(anu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from anukulan_b200 import pdhg
    lib = pdhg.lib()
    declared = _header_symbols()
    assert set(declared) == set(pdhg.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def test_library_version_and_no_fallback_without_device():
    from anukulan_b200 import pdhg
    assert "sm_100a" in pdhg.version()
    if pdhg.device_count() > 0:
        pytest.skip("a device is present")
    lp = lp_cases.standard(lp_cases.wyndor())
    with pytest.raises(pdhg.EngineError) as e:
        pdhg.solve_pdhg(lp)
    assert e.value.code == 3  # ANU_ERR_NO_DEVICE: no CPU fallback


@pytest.mark.parametrize("bad", [dict(tile_threads=64), dict(tile_threads=512),
                                 dict(cluster_chunks=2), dict(cluster_chunks=-1)])
def test_engine_options_validated_before_any_device_work(bad):
    """The C ABI checks the engine's own options first, with or without a
    device: an invalid tile size or cluster switch is ANU_ERR_INVALID."""
    from anukulan_b200 import pdhg
    lp = lp_cases.standard(lp_cases.wyndor())
    with pytest.raises(pdhg.EngineError) as e:
        pdhg.solve_pdhg(lp, max_iterations=10, **bad)
    assert e.value.code == 1
    assert next(iter(bad)) in str(e.value)


def test_struct_layout_roundtrip():
    # The C library writes its defaults into the ctypes struct; a layout
    # mismatch would scramble the fields checked above. Check sizes agree
    # with a field-by-field sum plus natural alignment.
    assert C.sizeof(abi.anu_pdhg_residual) == 12 * 8
    assert C.sizeof(abi.anu_pdhg_phases) == 6 * 8


@pytest.mark.skipif(not oracle.have_reference_b200(), reason="adapter build absent")
def test_reference_adapter_without_device_falls_back_and_fails_loudly():
    """Built with the adapter as anukulan::cuda_backend(), the reference keeps
    its own no-device behaviour: default_backend() is the CPU reference
    (backend.cpp:209-221), and asking for the device backend raises."""
    from anukulan_b200 import pdhg
    if pdhg.device_count() > 0:
        pytest.skip("a device is present")
    assert oracle.ref_b200_backend_name() == "cpu"
    lp = lp_cases.standard(lp_cases.wyndor())
    with pytest.raises(RuntimeError, match="no CUDA device"):
        oracle.ref_b200_solve(lp, tolerance=1e-6)
    for path in (oracle.REF_B200_TEST_BACKEND, oracle.REF_B200_TEST_PDHG):
        p = subprocess.run([path], capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stdout + p.stderr


def test_node_relaxation_rule():
    """NodeRelaxation judges a node as branch_and_bound.cpp:556-565 does:
    certified only when optimal and dual feasible to 1e-7 of the dual
    objective; the bound is then the dual objective."""
    from anukulan_b200.abi import PdhgResult, Residual
    from anukulan_b200.pdhg import NodeRelaxation

    def result(status, dual_objective, dual_inf):
        res = Residual(dual_residual_inf=dual_inf, dual_objective=dual_objective)
        return PdhgResult(status, np.zeros(1), np.zeros(1), 0.0, 0, 0, 0, 0, False, 0.0, 0.0,
                          0.0, 0.0, {}, res, (1.0, 1.0, 1.0, 1.0), 0, 0, 0.0, 0, "")

    ok = NodeRelaxation(result(abi.OPTIMAL, -2.0e6, 0.1))
    assert ok.optimal and ok.bound == -2.0e6 and not ok.proved_infeasible
    loose = NodeRelaxation(result(abi.OPTIMAL, -2.0e6, 0.3))
    assert not loose.optimal and np.isnan(loose.bound)
    small = NodeRelaxation(result(abi.OPTIMAL, 0.5, 1.0e-7))
    assert small.optimal and small.bound == 0.5
    assert not NodeRelaxation(result(abi.OPTIMAL, 0.5, 1.1e-7)).optimal
    inf = NodeRelaxation(result(abi.PRIMAL_INFEASIBLE, 0.0, 0.0))
    assert inf.proved_infeasible and not inf.optimal
    assert not NodeRelaxation(result(abi.ITERATION_LIMIT, 1.0, 0.0)).optimal


def test_node_relaxations_reject_bad_bounds():
    """Node bounds are (nodes x columns), the same shape for lower and
    upper; anything else is refused before the engine is asked."""
    from anukulan_b200.pdhg import solve_node_relaxations
    lp = lp_cases.standard(lp_cases.wyndor())
    n = lp.num_cols
    with pytest.raises(ValueError):
        solve_node_relaxations(lp, np.zeros((2, n)), np.ones((3, n)))
    with pytest.raises(ValueError):
        solve_node_relaxations(lp, np.zeros((2, n + 1)), np.ones((2, n + 1)))
