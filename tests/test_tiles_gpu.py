"""The single-LP product tile (options.tile_threads): 128 or 256 threads per
CTA for both products, or 0: an LP of at least 2^20 nonzeros gets short
trial solves of itself for each pair of tiles (K~ x, K~' y) at create, and
keeps the fastest pair; a smaller one takes 128.

Both tiles sum every row in the same order - a row of at most 32 nonzeros
serially by its thread, a longer one by a warp, a row longer than 1024 by a
CTA of its own over 128 strided lanes - so the tile changes timing only. The
tests hold every tile to bit-identical iterates, iteration and restart
counts, on LPs that reach all of those row classes:

- a power-law LP (row lengths 3 to 5000; its transpose has exactly 8
  nonzeros per row, the ELL kernel's shape), with and without the locality
  relabelling;
- an LP with a few very long rows among short ones (the long-row path);
- the full 200,000 x 300,000 power-law LP (2.4M nonzeros), where the
  trial solves run;
- a packed batch.
"""
import numpy as np
import pytest

import oracle
from anukulan_b200 import lpgen
from anukulan_b200.abi import ITERATION_LIMIT, OPTIMAL, PRECISION_FP32

pytestmark = pytest.mark.gpu

TILES = (128, 256, 0)


@pytest.fixture(scope="module")
def powerlaw():
    return lpgen.power_law_lp(m=20_000, n=30_000)[0]


@pytest.fixture(scope="module")
def long_rows():
    # Three rows of 2,500 nonzeros among rows of about 9.
    return lpgen.long_row_stack(m=2000, n=3000, long_len=2500).case(0)


def same(a, b):
    return (a.status == b.status and a.iterations == b.iterations
            and a.restarts == b.restarts and np.array_equal(a.x, b.x)
            and np.array_equal(a.y, b.y))


def test_powerlaw_reaches_every_row_class(powerlaw):
    lengths = powerlaw.k.row_lengths()
    assert lengths.min() <= 32 and ((lengths > 32) & (lengths <= 1024)).any()
    assert (lengths > 1024).any()
    assert np.all(np.diff(powerlaw.k.start) >= 0)


@pytest.mark.parametrize("precision", [0, PRECISION_FP32])
@pytest.mark.parametrize("locality_order", [0, 1])
def test_tiles_bit_identical_fixed_budget(engine, powerlaw, precision, locality_order):
    kw = dict(max_iterations=600, polish_on_exit=0, polish_feasibility=0,
              precision=precision, locality_order=locality_order)
    runs = [engine.solve_pdhg(powerlaw, tile_threads=t, **kw) for t in TILES]
    assert runs[0].status == ITERATION_LIMIT and runs[0].iterations == 600
    for t, r in zip(TILES[1:], runs[1:]):
        assert same(runs[0], r), t


@pytest.mark.parametrize("precision", [0, PRECISION_FP32])
def test_tiles_bit_identical_to_tolerance(engine, powerlaw, precision):
    runs = [engine.solve_pdhg(powerlaw, tolerance=1e-4, precision=precision, tile_threads=t)
            for t in TILES]
    assert runs[0].status == OPTIMAL, runs[0].message
    for t, r in zip(TILES[1:], runs[1:]):
        assert same(runs[0], r), t
    assert oracle.oracle_residual(powerlaw, runs[0].x, runs[0].y).converged(1e-4)


@pytest.mark.parametrize("precision", [0, PRECISION_FP32])
def test_tiles_bit_identical_long_rows(engine, long_rows, precision):
    assert long_rows.k.row_lengths().max() > 1024
    kw = dict(max_iterations=400, polish_on_exit=0, polish_feasibility=0, precision=precision)
    runs = [engine.solve_pdhg(long_rows, tile_threads=t, **kw) for t in TILES]
    for t, r in zip(TILES[1:], runs[1:]):
        assert same(runs[0], r), t
    if precision == 0:
        o = oracle.oracle_solve(long_rows, **kw)
        assert runs[0].iterations == o.iterations and runs[0].restarts == o.restarts
        scale = max(1.0, float(np.max(np.abs(o.x))))
        assert float(np.max(np.abs(runs[0].x - o.x))) / scale < 1e-10


@pytest.fixture(scope="module")
def powerlaw_full():
    return lpgen.power_law_lp()[0]


@pytest.mark.parametrize("precision", [0, PRECISION_FP32])
def test_trial_tuned_tiles_bit_identical(engine, powerlaw_full, precision):
    """At full size tile_threads=0 runs the trial solves; whatever pair they
    choose, the solve that follows equals the fixed-tile ones bit for bit."""
    kw = dict(max_iterations=300, polish_on_exit=0, polish_feasibility=0, precision=precision)
    runs = {t: engine.solve_pdhg(powerlaw_full, tile_threads=t, **kw) for t in TILES}
    tuned = runs[0]
    assert tuned.tile_trial_seconds > 0.0
    assert tuned.row_product_threads in (128, 256)
    assert tuned.column_product_threads in (128, 256)
    for t in (128, 256):
        assert runs[t].tile_trial_seconds == 0.0
        assert runs[t].row_product_threads == runs[t].column_product_threads == t
        assert same(tuned, runs[t]), t
    assert tuned.iterations == 300


def test_small_lp_takes_default_tile(engine, powerlaw):
    r = engine.solve_pdhg(powerlaw, max_iterations=40, tile_threads=0)
    assert r.tile_trial_seconds == 0.0
    assert r.row_product_threads == r.column_product_threads == 128


def test_packed_tiles_bit_identical(engine):
    lps = [lp for lp, _ in lpgen.packed_batch(count=12, min_rows=300, max_rows=20_000, seed=78)]
    kw = dict(tolerance=1e-6, precision=PRECISION_FP32)
    fixed = {t: engine.solve_packed(lps, tile_threads=t, **kw) for t in (128, 256)}
    tuned = engine.solve_packed(lps, tile_threads=0, **kw)
    chosen = tuned[0].row_product_threads
    assert chosen in (128, 256)
    for t in (128, 256):
        assert all(r.row_product_threads == r.column_product_threads == t for r in fixed[t])
    for k, (a, b, c) in enumerate(zip(fixed[128], fixed[256], tuned)):
        assert c.row_product_threads == chosen, k
        assert same(a, b) and same(a, c), k


def test_invalid_tile_rejected(engine, powerlaw):
    with pytest.raises(Exception, match="tile_threads"):
        engine.solve_pdhg(powerlaw, tile_threads=64, max_iterations=10)
