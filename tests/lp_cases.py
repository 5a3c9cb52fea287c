"""Known-answer LPs of the PDHG path.

The reference pins its solver on small textbook LPs with known optima
(tests/test_pdhg.cpp:48-470 in anukulan). They are restated here as models so
the oracle and the engine can be checked against the same answers:

  wyndor          max 3x + 5y, x <= 4, 2y <= 12, 3x + 2y <= 18  -> 36 at (2, 6)
  equalities      min x + y, x + y = 10, x - y = 2              -> 10 at (6, 4)
  boxed_free      min -x - y, x + y <= 10, 1 <= x <= 3, y free  -> -10
  range_row       min x + 2y, 5 <= x + y <= 8                   -> 5 at (5, 0)
  degenerate      max x + y, x + y <= 2, x <= 1, y <= 1         -> 2 at (1, 1)
  offset          min x + 7, x >= 4                             -> 11
  norm_4          rows 3x >= 1, 4y >= 1 (||K|| = 4 by inspection)
  empty_rows      a row with no coefficients; x in [0,5] cost 1, y in [0,5]
                  cost -1                                        -> -5 at (0, 5)
  infeasible      x + y = 1, x + y = 3, x, y >= 0 (no feasible point)
"""
from __future__ import annotations

import numpy as np

from anukulan_b200.model import Csr, Model, StandardLp, to_standard_form

INF = float("inf")


def _model(rows, cols, entries, obj, row_lo, row_hi, col_lo, col_hi, maximize=False,
           offset=0.0, name=""):
    r = [e[0] for e in entries]
    c = [e[1] for e in entries]
    v = [e[2] for e in entries]
    a = Csr.from_triplets(rows, cols, r, c, v)
    return Model(a, np.array(obj, float), np.array(row_lo, float), np.array(row_hi, float),
                 np.array(col_lo, float), np.array(col_hi, float), maximize, offset, name)


def standard(model: Model) -> StandardLp:
    sf = to_standard_form(model)
    assert sf.ok, sf.error
    return sf.lp


def wyndor() -> Model:
    return _model(3, 2, [(0, 0, 1.0), (2, 0, 3.0), (1, 1, 2.0), (2, 1, 2.0)], [3.0, 5.0],
                  [-INF] * 3, [4.0, 12.0, 18.0], [0, 0], [INF, INF], maximize=True,
                  name="wyndor")


def equalities() -> Model:
    return _model(2, 2, [(0, 0, 1.0), (1, 0, 1.0), (0, 1, 1.0), (1, 1, -1.0)], [1.0, 1.0],
                  [10.0, 2.0], [10.0, 2.0], [0, 0], [INF, INF], name="equalities")


def boxed_free() -> Model:
    return _model(1, 2, [(0, 0, 1.0), (0, 1, 1.0)], [-1.0, -1.0], [-INF], [10.0],
                  [1.0, -INF], [3.0, INF], name="boxed_free")


def range_row() -> Model:
    return _model(1, 2, [(0, 0, 1.0), (0, 1, 1.0)], [1.0, 2.0], [5.0], [8.0], [0, 0],
                  [INF, INF], name="range_row")


def degenerate() -> Model:
    return _model(3, 2, [(0, 0, 1.0), (1, 0, 1.0), (0, 1, 1.0), (2, 1, 1.0)], [1.0, 1.0],
                  [-INF] * 3, [2.0, 1.0, 1.0], [0, 0], [INF, INF], maximize=True,
                  name="degenerate")


def offset() -> Model:
    return _model(1, 1, [(0, 0, 1.0)], [1.0], [4.0], [INF], [0.0], [INF], offset=7.0,
                  name="offset")


def norm_4() -> Model:
    return _model(2, 2, [(0, 0, 3.0), (1, 1, 4.0)], [1.0, 1.0], [1.0, 1.0], [INF, INF],
                  [0, 0], [INF, INF], name="norm_4")


def empty_rows() -> Model:
    return _model(1, 2, [], [1.0, -1.0], [-1.0], [INF], [0.0, 0.0], [5.0, 5.0],
                  name="empty_rows")


def infeasible() -> Model:
    return _model(2, 2, [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 1.0)], [1.0, 1.0],
                  [1.0, 3.0], [1.0, 3.0], [0, 0], [INF, INF], name="infeasible")


# (builder, known objective, known x or None)
KNOWN = {
    "wyndor": (wyndor, 36.0, [2.0, 6.0]),
    "equalities": (equalities, 10.0, [6.0, 4.0]),
    "boxed_free": (boxed_free, -10.0, None),
    "range_row": (range_row, 5.0, None),
    "degenerate": (degenerate, 2.0, [1.0, 1.0]),
    "offset": (offset, 11.0, None),
}
