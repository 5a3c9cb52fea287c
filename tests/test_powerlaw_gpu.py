"""The 200,000 x 300,000 power-law LP (2.4M nonzeros, row lengths drawn from
a power law with exponent 2.2 on [3, 5000], 8 nonzeros per column) at full
size, through the C ABI.

- FP64 iterates after a fixed number of iterations match the oracle (the
  restated reference solve_pdhg) to 1e-10 relative, with the same restart
  count. At this size the oracle's serial FP64 iteration takes a few
  seconds per hundred iterations, so the check stops at 200.
- FP32 iterates with FP64 checks and refinement reach relative KKT 1e-4;
  the oracle re-evaluates the returned point in FP64, and the objective is
  compared with the planted optimum c'x0 of the generator.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def powerlaw():
    return lpgen.power_law_lp()


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def test_powerlaw_shape(powerlaw):
    lp, _ = powerlaw
    lengths = lp.k.row_lengths()
    assert (lp.num_rows, lp.num_cols, lp.k.nnz) == (200_000, 300_000, 2_400_000)
    assert lengths.min() >= 3 and lengths.max() <= 5000


def test_powerlaw_fp64_iterates_match_oracle(engine, powerlaw):
    lp, _ = powerlaw
    kw = dict(max_iterations=200, polish_on_exit=0, polish_feasibility=0)
    r = engine.solve_pdhg(lp, **kw)
    o = oracle.oracle_solve(lp, **kw)
    assert r.status == o.status == ITERATION_LIMIT
    assert r.iterations == o.iterations == 200
    assert r.restarts == o.restarts
    assert rel_err(r.x, o.x) < 1e-10
    assert rel_err(r.y, o.y) < 1e-10


def test_powerlaw_fp32_refined_reaches_1e4(engine, powerlaw):
    lp, objective = powerlaw
    r = engine.solve_pdhg(lp, tolerance=1e-4, precision=PRECISION_FP32, max_iterations=400_000)
    assert r.status == OPTIMAL, r.message
    res = oracle.oracle_residual(lp, r.x, r.y)
    assert res.converged(1e-4), res
    assert abs(r.objective - objective) <= 1e-3 * abs(objective)


# ------------------------------------------------------------ column slabs
# FP32 single-LP products over this matrix (and its transpose) gather from
# column slabs staged in shared memory (slab_kernel). Checked directly,
# through anu_spmv_fp32, against the FP64 product: each row's error within
# 1e-5 of the row's sum of |a_ij x_j| (FP32 rounding of sums of up to
# ~5,000 terms), and against the row-block kernel it replaces.

def _abs_bound(a, x):
    import scipy.sparse as sp
    A = sp.csr_matrix((a.value, a.index, a.start), shape=(a.rows, a.cols))
    return A @ x, abs(A) @ np.abs(x)


@pytest.mark.parametrize("side", ["k", "kt"])
def test_slab_product_matches_fp64(engine, powerlaw, side):
    lp, _ = powerlaw
    a = lp.k if side == "k" else lp.k.transpose()
    rng = np.random.default_rng(17)
    x = rng.standard_normal(a.cols).astype(np.float32)
    ref, mag = _abs_bound(a, x.astype(np.float64))
    ys, used = engine.spmv_fp32(a, x, engine.SPMV_SLABS)
    assert used == engine.SPMV_SLABS
    yr, used_r = engine.spmv_fp32(a, x, engine.SPMV_ROWS)
    assert used_r == engine.SPMV_ROWS
    _, used_auto = engine.spmv_fp32(a, x)
    assert used_auto == engine.SPMV_SLABS
    err_s = float(np.max(np.abs(ys - ref) / np.maximum(mag, 1e-30)))
    err_r = float(np.max(np.abs(yr - ref) / np.maximum(mag, 1e-30)))
    assert err_s <= 1e-5, err_s
    assert err_r <= 1e-5, err_r
    # Deterministic: the same inputs give the same bits.
    again, _ = engine.spmv_fp32(a, x, engine.SPMV_SLABS)
    assert np.array_equal(again, ys)


def test_slab_product_ragged_rows(engine):
    # Empty rows, rows of a few nonzeros and rows of thousands (summed by
    # whole warps inside a unit), several long rows to a unit, 150,000
    # columns in 4 slabs.
    from anukulan_b200.model import Csr
    rng = np.random.default_rng(5)
    rows, cols = 1500, 150_000
    lengths = rng.choice([0, 0, 1, 3, 17, 40, 300, 2500, 7000], size=rows)
    lengths[:4] = [7000, 0, 6500, 1]
    start = np.zeros(rows + 1, np.int64)
    start[1:] = np.cumsum(lengths)
    index = np.concatenate([np.sort(rng.choice(cols, size=int(L), replace=False))
                            for L in lengths]).astype(np.int32)
    value = rng.uniform(-1.0, 1.0, size=index.size)
    a = Csr(rows, cols, start.astype(np.int32), index, value)
    assert a.nnz >= 1 << 20
    x = rng.standard_normal(cols).astype(np.float32)
    ref, mag = _abs_bound(a, x.astype(np.float64))
    ys, used = engine.spmv_fp32(a, x, engine.SPMV_SLABS)
    assert used == engine.SPMV_SLABS
    assert np.all(ys[lengths == 0] == 0.0)
    err = float(np.max(np.abs(ys - ref) / np.maximum(mag, 1e-30)))
    assert err <= 1e-5, err


def test_slab_product_not_taken_by_small_matrix(engine):
    lp, _ = lpgen.random_lp()
    x = np.ones(lp.num_cols, np.float32)
    y, used = engine.spmv_fp32(lp.k, x)
    assert used == engine.SPMV_ROWS
    with pytest.raises(engine.EngineError):
        engine.spmv_fp32(lp.k, x, engine.SPMV_SLABS)


def test_slab_iterations_track_row_blocks(engine, powerlaw):
    # 200 FP32 iterations with refinement, slabs on and off: the same
    # restarts, and iterates that differ only by FP32 rounding of the sums.
    lp, _ = powerlaw
    kw = dict(max_iterations=200, polish_on_exit=0, polish_feasibility=0,
              precision=PRECISION_FP32)
    s = engine.solve_pdhg(lp, slab_products=1, **kw)
    r = engine.solve_pdhg(lp, slab_products=0, **kw)
    assert s.iterations == r.iterations == 200
    assert s.restarts == r.restarts
    dx, dy = rel_err(s.x, r.x), rel_err(s.y, r.y)
    print(f"slab vs row blocks after 200 FP32 iterations: x {dx:.3e}, y {dy:.3e}")
    assert dx < 1e-5 and dy < 1e-5, (dx, dy)
