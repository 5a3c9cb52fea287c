"""Seeded synthetic LPs for the five workloads of the PDHG path.

Every generator takes a seed and returns standard-form LPs
(:class:`~anukulan_b200.model.StandardLp`). The constructions:

* :func:`random_lp` - the known-optimum sparse LP. Each column of A gets 8
  distinct uniformly random rows with N(0,1) values; x0 ~ U(0,10) with 30% of
  entries set to 0; b = A x0; y0 ~ N(0,1); reduced costs s = |N(0,1)| on the
  zero entries of x0 and 0 elsewhere; c = A'y0 + s; bounds [0, 10]; all rows
  equalities. (x0, y0) satisfies the KKT conditions, so the optimum is
  c'x0 = b'y0 whatever solver is asked.
* :func:`power_law_lp` - the same construction with row lengths drawn from a
  discrete power law P(L) ~ L^-2.2 on [3, 5000], fixed to an exact nonzero
  total, and rows assigned to columns by a configuration model (each row listed
  L times, shuffled, cut into columns of 8, duplicates in a column repaired by
  swapping slots with other columns).
* :func:`refinery_stack` - a multiperiod refinery-shaped planning LP (24
  period blocks of 115 rows x 160 columns, yields U(0.2, 1.5), capacity rows
  with rhs U(50, 500), inventory-linking equality rows between consecutive
  periods) and 60 what-if cases that each change the base in one place, in the
  manner of the reference's scripts/refinery_cases.py:36-50 (crude price
  -6/-3/+3/+6 %, a crude supply halved, a product demand -/+10 %, a unit
  capacity cut 20 % in one of periods 1-4). Buying nothing is feasible, so no
  case is infeasible.
* :func:`packed_batch` - 256 independent :func:`random_lp` problems with row
  counts log-uniform in [500, 50000] and 1.5x as many columns.
* :func:`adjoint_case` - the refinery base with a held-out price vector
  c_hat = c * (1 + 0.05 N(0,1)).

Seeds default to 20261203 + workload index.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

from .model import Csr, Model, StandardLp, to_standard_form

INF = float("inf")
BASE_SEED = 20261203


def _kkt_lp(a: Csr, rng: np.random.Generator, name: str) -> Tuple[StandardLp, float]:
    """Builds b, c from a known primal-dual optimum (x0, y0); returns the LP
    and c'x0."""
    m, n = a.rows, a.cols
    x0 = rng.uniform(0.0, 10.0, n)
    zero = rng.random(n) < 0.3
    x0[zero] = 0.0
    y0 = rng.standard_normal(m)
    s = np.where(zero, np.abs(rng.standard_normal(n)), 0.0)
    b = a.multiply(x0)
    c = a.transpose().multiply(y0) + s
    lp = StandardLp(a, c, b, np.zeros(n), np.full(n, 10.0), m, 1.0, 0.0,
                    np.arange(m, dtype=np.int32), np.ones(m), name)
    return lp, float(np.dot(c, x0))


def random_lp(m: int = 1000, n: int = 1500, per_col: int = 8,
              seed: int = BASE_SEED + 0) -> Tuple[StandardLp, float]:
    """Known-optimum LP with `per_col` distinct uniformly random rows per column.
    Returns (lp, c'x0)."""
    rng = np.random.default_rng(seed)
    per_col = min(per_col, m)
    # Distinct rows per column: argsort of uniform keys, first per_col.
    rows = np.empty((n, per_col), dtype=np.int64)
    chunk = max(1, (1 << 22) // max(m, 1))
    for j0 in range(0, n, chunk):
        j1 = min(n, j0 + chunk)
        keys = rng.random((j1 - j0, m))
        rows[j0:j1] = np.argpartition(keys, per_col - 1, axis=1)[:, :per_col]
    vals = rng.standard_normal((n, per_col))
    cols = np.repeat(np.arange(n, dtype=np.int64), per_col)
    a = Csr.from_triplets(m, n, rows.reshape(-1), cols, vals.reshape(-1))
    return _kkt_lp(a, rng, f"random_{m}x{n}")


def power_law_row_lengths(m: int, total: int, rng: np.random.Generator,
                          exponent: float = 2.2, lmin: int = 3,
                          lmax: int = 5000) -> np.ndarray:
    """Row lengths from P(L) ~ L^-exponent on [lmin, lmax], then single slots
    added to or removed from random rows (staying inside [lmin, lmax]) until
    they sum to `total` exactly. Lengths are never rescaled."""
    support = np.arange(lmin, lmax + 1, dtype=np.int64)
    p = support.astype(np.float64) ** (-exponent)
    p /= p.sum()
    lengths = rng.choice(support, size=m, p=p)
    diff = int(total - lengths.sum())
    while diff != 0:
        step = 1 if diff > 0 else -1
        picks = rng.integers(0, m, size=min(abs(diff), m))
        for i in picks.tolist():
            if diff == 0:
                break
            nv = lengths[i] + step
            if lmin <= nv <= lmax:
                lengths[i] = nv
                diff -= step
    return lengths


def power_law_lp(m: int = 200_000, n: int = 300_000, per_col: int = 8,
                 seed: int = BASE_SEED + 1) -> Tuple[StandardLp, float]:
    """Known-optimum LP whose row lengths follow a power law (exponent 2.2,
    max 5000) and whose columns hold exactly `per_col` nonzeros. Returns
    (lp, c'x0)."""
    rng = np.random.default_rng(seed)
    total = n * per_col
    lengths = power_law_row_lengths(m, total, rng)
    slots = np.repeat(np.arange(m, dtype=np.int64), lengths)
    rng.shuffle(slots)
    grid = slots.reshape(n, per_col)
    # Repair duplicate rows inside a column by swapping the offending slot
    # with a random slot of a random other column; repeat until none remain.
    for _ in range(1000):
        srt = np.sort(grid, axis=1)
        dup_cols = np.nonzero((srt[:, 1:] == srt[:, :-1]).any(axis=1))[0]
        if dup_cols.size == 0:
            break
        for j in dup_cols.tolist():
            row = grid[j]
            seen = set()
            for s in range(per_col):
                v = int(row[s])
                if v in seen:
                    while True:
                        j2 = int(rng.integers(0, n))
                        s2 = int(rng.integers(0, per_col))
                        v2 = int(grid[j2, s2])
                        if j2 != j and v2 not in seen and v not in set(grid[j2].tolist()):
                            grid[j, s], grid[j2, s2] = v2, v
                            v = v2
                            break
                seen.add(v)
    else:
        raise RuntimeError("duplicate repair did not converge")
    vals = rng.standard_normal((n, per_col))
    cols = np.repeat(np.arange(n, dtype=np.int64), per_col)
    a = Csr.from_triplets(m, n, grid.reshape(-1), cols, vals.reshape(-1))
    return _kkt_lp(a, rng, f"powerlaw_{m}x{n}")


# --------------------------------------------------------------- refinery


@dataclass
class RefineryLayout:
    periods: int
    rows_per_period: int
    cols_per_period: int
    crudes: int
    products: int
    # column offsets inside a period
    buy: int
    sell: int
    inv: int
    process: int
    # row offsets inside a period (model order)
    balance: int
    crude_rows: int
    demand: int
    capacity: int


def refinery_layout(periods: int = 24) -> RefineryLayout:
    return RefineryLayout(periods=periods, rows_per_period=115, cols_per_period=160,
                          crudes=8, products=4, buy=0, sell=8, inv=12, process=16,
                          balance=0, crude_rows=4, demand=12, capacity=16)


def refinery_model(periods: int = 24, seed: int = BASE_SEED + 2) -> Tuple[Model, RefineryLayout]:
    """The base refinery-shaped planning model (before the standard form).

    Per period t (160 columns, 115 rows):
      columns  BUY_c (8 crudes, cost U(50,80), supply ceiling U(200,800)),
               SELL_p (4 products, revenue U(90,130) as a negative cost),
               INV_p (4 inventories carried into t+1, cost U(0.5,2), cap 1000),
               144 process columns (operating cost U(1,10)), each consuming one
               or two crudes and yielding one to three products with
               coefficients U(0.2,1.5) and sitting in about 9 capacity rows;
      rows     4 product balances (inventory-linking equalities, rhs 0):
                 production + INV_{t-1} - SELL - INV_t = 0,
               8 crude balances  BUY_c - consumption >= 0,
               4 demands SELL_p <= D (U(50,500)),
               99 capacity rows <= U(50,500) (rows 0-2 are the CDU, FCC and
               HDT analogues the outage cases cut).
    """
    L = refinery_layout(periods)
    rng = np.random.default_rng(seed)
    T = periods
    nc = L.cols_per_period
    nr = L.rows_per_period
    n = T * nc
    m = T * nr
    crude_cost = rng.uniform(50.0, 80.0, L.crudes)
    supply = rng.uniform(200.0, 800.0, L.crudes)
    price = rng.uniform(90.0, 130.0, L.products)
    hold = rng.uniform(0.5, 2.0, L.products)
    nproc = nc - L.process
    ncap = nr - L.capacity
    # Process structure shared by every period (the same plant each period).
    proc_crudes = [rng.choice(L.crudes, size=rng.integers(1, 3), replace=False)
                   for _ in range(nproc)]
    proc_products = [rng.choice(L.products, size=rng.integers(1, 4), replace=False)
                     for _ in range(nproc)]
    proc_caps = [rng.choice(ncap, size=rng.integers(7, 12), replace=False)
                 for _ in range(nproc)]
    proc_cost = rng.uniform(1.0, 10.0, nproc)

    rr, cc, vv = [], [], []
    obj = np.zeros(n)
    col_lo = np.zeros(n)
    col_hi = np.full(n, INF)
    row_lo = np.zeros(m)
    row_hi = np.zeros(m)

    def add(r, c, v):
        rr.append(r)
        cc.append(c)
        vv.append(v)

    for t in range(T):
        c0 = t * nc
        r0 = t * nr
        for k in range(L.crudes):
            col = c0 + L.buy + k
            obj[col] = crude_cost[k]
            col_hi[col] = supply[k]
            add(r0 + L.crude_rows + k, col, 1.0)
        for p in range(L.products):
            col = c0 + L.sell + p
            obj[col] = -price[p]
            add(r0 + L.balance + p, col, -1.0)
            add(r0 + L.demand + p, col, 1.0)
            inv = c0 + L.inv + p
            obj[inv] = hold[p]
            col_hi[inv] = 1000.0
            add(r0 + L.balance + p, inv, -1.0)
            if t + 1 < T:  # inventory enters the next period's balance
                add(r0 + nr + L.balance + p, inv, 1.0)
        for a in range(nproc):
            col = c0 + L.process + a
            obj[col] = proc_cost[a]
            for k in proc_crudes[a]:
                add(r0 + L.crude_rows + int(k), col, -rng.uniform(0.2, 1.5))
            for p in proc_products[a]:
                add(r0 + L.balance + int(p), col, rng.uniform(0.2, 1.5))
            for cap in proc_caps[a]:
                add(r0 + L.capacity + int(cap), col, rng.uniform(0.2, 1.5))
        # row bounds
        for p in range(L.products):
            row_lo[r0 + L.balance + p] = 0.0
            row_hi[r0 + L.balance + p] = 0.0
        for k in range(L.crudes):
            row_lo[r0 + L.crude_rows + k] = 0.0
            row_hi[r0 + L.crude_rows + k] = INF
        for p in range(L.products):
            row_lo[r0 + L.demand + p] = -INF
            row_hi[r0 + L.demand + p] = rng.uniform(50.0, 500.0)
        for cap in range(ncap):
            row_lo[r0 + L.capacity + cap] = -INF
            row_hi[r0 + L.capacity + cap] = rng.uniform(50.0, 500.0)
    a = Csr.from_triplets(m, n, rr, cc, vv)
    model = Model(a, obj, row_lo, row_hi, col_lo, col_hi, False, 0.0, f"refinery_{T}")
    return model, L


def refinery_cases(layout: RefineryLayout) -> List[Tuple[str, str, int, float, int]]:
    """(name, kind, subject, factor, period) of the 60 what-if cases."""
    out = []
    for k in range(layout.crudes):
        for pct in (-6, -3, 3, 6):
            out.append((f"price_crude{k}_{pct:+d}", "price", k, 1.0 + pct / 100.0, -1))
    for k in range(layout.crudes):
        out.append((f"supply_crude{k}_half", "supply", k, 0.5, -1))
    for p in range(layout.products):
        for pct in (-10, 10):
            out.append((f"demand_product{p}_{pct:+d}", "demand", p, 1.0 + pct / 100.0, -1))
    for unit, factor in ((0, 0.8), (1, 0.8), (2, 0.8)):
        for period in (1, 2, 3, 4):
            out.append((f"outage_unit{unit}_p{period}", "capacity", unit, factor, period))
    return out


def apply_case(model: Model, layout: RefineryLayout, kind: str, subject: int,
               factor: float, period: int) -> Model:
    obj = model.objective.copy()
    col_hi = model.col_upper.copy()
    row_hi = model.row_upper.copy()
    nc, nr = layout.cols_per_period, layout.rows_per_period
    if kind == "price":
        for t in range(layout.periods):
            obj[t * nc + layout.buy + subject] *= factor
    elif kind == "supply":
        for t in range(layout.periods):
            col_hi[t * nc + layout.buy + subject] *= factor
    elif kind == "demand":
        for t in range(layout.periods):
            row_hi[t * nr + layout.demand + subject] *= factor
    elif kind == "capacity":
        t = period - 1
        row_hi[t * nr + layout.capacity + subject] *= factor
    else:
        raise ValueError(kind)
    return Model(model.constraints, obj, model.row_lower, row_hi, model.col_lower,
                 col_hi, model.maximize, model.objective_offset, model.name)


@dataclass
class CaseStack:
    base: StandardLp
    names: List[str]
    c: np.ndarray      # K x n
    q: np.ndarray      # K x m
    lower: np.ndarray  # K x n
    upper: np.ndarray  # K x n

    @property
    def num_cases(self) -> int:
        return len(self.names)

    def case(self, k: int) -> StandardLp:
        return self.base.with_vectors(self.c[k], self.q[k], self.lower[k], self.upper[k])


def refinery_stack(periods: int = 24, seed: int = BASE_SEED + 2) -> CaseStack:
    """The base refinery LP in standard form and its 60 cases. Every case has
    the base's matrix exactly (only c, q and bounds move)."""
    model, L = refinery_model(periods, seed)
    base = to_standard_form(model)
    assert base.ok, base.error
    names, cs, qs, los, his = [], [], [], [], []
    for name, kind, subject, factor, period in refinery_cases(L):
        sf = to_standard_form(apply_case(model, L, kind, subject, factor, period))
        assert sf.ok, sf.error
        assert np.array_equal(sf.lp.k.index, base.lp.k.index)
        assert np.array_equal(sf.lp.k.value, base.lp.k.value)
        names.append(name)
        cs.append(sf.lp.c)
        qs.append(sf.lp.q)
        los.append(sf.lp.lower)
        his.append(sf.lp.upper)
    return CaseStack(base.lp, names, np.stack(cs), np.stack(qs), np.stack(los),
                     np.stack(his))


def sparse_random_lp(m: int, n: int, per_col: int = 8,
                     seed: int = BASE_SEED) -> Tuple[StandardLp, float]:
    """The construction of :func:`random_lp` (per column `per_col` distinct
    uniformly random rows, N(0,1) values, planted optimum) with a sampler
    whose cost is linear in the nonzeros: draw every slot at random, then
    redraw the slots that repeat a row of their column until none do."""
    rng = np.random.default_rng(seed)
    per_col = min(per_col, m)
    rows = rng.integers(0, m, size=(n, per_col))
    while True:
        srt = np.sort(rows, axis=1)
        dup_cols = np.nonzero((srt[:, 1:] == srt[:, :-1]).any(axis=1))[0]
        if dup_cols.size == 0:
            break
        sub = rows[dup_cols]
        first = np.ones_like(sub, dtype=bool)
        for s in range(1, per_col):
            first[:, s] = ~(sub[:, :s] == sub[:, s:s + 1]).any(axis=1)
        redraw = ~first
        sub[redraw] = rng.integers(0, m, size=int(redraw.sum()))
        rows[dup_cols] = sub
    vals = rng.standard_normal((n, per_col))
    cols = np.repeat(np.arange(n, dtype=np.int64), per_col)
    a = Csr.from_triplets(m, n, rows.reshape(-1), cols, vals.reshape(-1))
    return _kkt_lp(a, rng, f"sparse_random_{m}x{n}")


def long_row_stack(m: int = 600, n: int = 900, per_col: int = 6, long_rows: int = 3,
                   long_len: int = 700, cases: int = 20,
                   seed: int = BASE_SEED + 5) -> CaseStack:
    """A stack of `cases` known-optimum LPs sharing one matrix that mixes
    `per_col` random rows per column with `long_rows` rows of `long_len`
    nonzeros (longer than eight 32-nonzero segments). Cases differ in c."""
    rng = np.random.default_rng(seed)
    rows = np.concatenate([rng.integers(long_rows, m, size=n * per_col),
                           np.repeat(np.arange(long_rows), long_len)])
    cols = np.concatenate([np.repeat(np.arange(n), per_col),
                           np.concatenate([rng.choice(n, long_len, replace=False)
                                           for _ in range(long_rows)])])
    vals = rng.standard_normal(rows.size)
    key = rows.astype(np.int64) * n + cols
    _, first = np.unique(key, return_index=True)
    a = Csr.from_triplets(m, n, rows[first], cols[first], vals[first])
    lp, _ = _kkt_lp(a, rng, f"long_rows_{m}x{n}")
    c = lp.c[None, :] * (1.0 + 0.05 * rng.standard_normal((cases, n)))
    return CaseStack(lp, [f"long_rows_case{k}" for k in range(cases)], c,
                     np.repeat(lp.q[None, :], cases, 0), np.repeat(lp.lower[None, :], cases, 0),
                     np.repeat(lp.upper[None, :], cases, 0))


def packed_batch(count: int = 256, seed: int = BASE_SEED + 3,
                 min_rows: int = 500, max_rows: int = 50_000) -> List[Tuple[StandardLp, float]]:
    """`count` independent known-optimum LPs, rows log-uniform in
    [min_rows, max_rows], 1.5x as many columns, 8 nonzeros per column."""
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(min_rows), np.log(max_rows), count)).astype(np.int64)
    out = []
    for i, mi in enumerate(rows.tolist()):
        out.append(sparse_random_lp(int(mi), int(round(1.5 * mi)), 8, seed * 1000 + i))
    return out


def adjoint_case(periods: int = 24, seed: int = BASE_SEED + 4) -> Tuple[CaseStack, np.ndarray]:
    """The refinery stack and a held-out price vector c_hat = c (1 + 0.05 N(0,1))
    of the base, for the unrolled-PDHG sensitivity workload."""
    stack = refinery_stack(periods, BASE_SEED + 2)
    rng = np.random.default_rng(seed)
    c_hat = stack.base.c * (1.0 + 0.05 * rng.standard_normal(stack.base.num_cols))
    return stack, c_hat
