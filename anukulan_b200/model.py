"""Host-side data model of the PDHG path: models, CSR matrices and the
standard form the engine solves.

Restates, in numpy, the reference's

  * ``SparseMatrix::from_triplets`` (src/anukulan/sparse.cpp:24-69): duplicates
    summed, exact zeros dropped, columns sorted within each row;
  * ``SparseMatrix::transpose`` (src/anukulan/sparse.cpp:93-117);
  * ``Model`` (src/anukulan/model.hpp:23-49), row/column bound form;
  * ``to_standard_form`` (src/anukulan/standard_form.cpp:72-165): equalities
    first, two-sided rows split into ``a'x >= lo`` and ``-a'x >= -hi``,
    rows without a finite bound dropped, ``row_origin`` recorded;
  * ``StandardLp`` (src/anukulan/standard_form.hpp:23-66).

The integer maps (``row_origin`` and the CSR structure) are bit-exact with the
reference; the tests pin them against the reference's own build.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

INF = float("inf")


@dataclass
class Csr:
    """CSR with int32 indices and float64 values (``SparseMatrix``)."""

    rows: int
    cols: int
    start: np.ndarray  # int32, rows + 1
    index: np.ndarray  # int32, nnz
    value: np.ndarray  # float64, nnz

    @property
    def nnz(self) -> int:
        return int(self.index.shape[0])

    @staticmethod
    def from_triplets(rows: int, cols: int, r, c, v) -> "Csr":
        """``SparseMatrix::from_triplets`` (sparse.cpp:24-69)."""
        r = np.asarray(r, dtype=np.int64)
        c = np.asarray(c, dtype=np.int64)
        v = np.asarray(v, dtype=np.float64)
        if r.size == 0:
            return Csr(rows, cols, np.zeros(rows + 1, np.int32),
                       np.zeros(0, np.int32), np.zeros(0, np.float64))
        if r.min() < 0 or r.max() >= rows or c.min() < 0 or c.max() >= cols:
            raise ValueError("triplet index out of range")
        # Stable order (row, col, original position): duplicates are summed in
        # input order, which is the order the reference's counting sort keeps.
        key = r * cols + c
        order = np.argsort(key, kind="stable")
        key = key[order]
        v = v[order]
        first = np.ones(key.size, dtype=bool)
        first[1:] = key[1:] != key[:-1]
        group = np.cumsum(first) - 1
        # Sequential left-to-right summation per group, as the reference does.
        sums = np.zeros(int(group[-1]) + 1, dtype=np.float64)
        if np.all(first):
            sums = v.copy()
        else:
            for g, val in zip(group.tolist(), v.tolist()):
                sums[g] += val
        ukey = key[first]
        keep = sums != 0.0
        ukey = ukey[keep]
        sums = sums[keep]
        rr = (ukey // cols).astype(np.int64)
        cc = (ukey % cols).astype(np.int32)
        start = np.zeros(rows + 1, dtype=np.int64)
        np.add.at(start, rr + 1, 1)
        start = np.cumsum(start).astype(np.int32)
        return Csr(rows, cols, start, cc, sums)

    def transpose(self) -> "Csr":
        """``SparseMatrix::transpose`` (sparse.cpp:93-117)."""
        rows_of = np.repeat(np.arange(self.rows, dtype=np.int64),
                            np.diff(self.start.astype(np.int64)))
        order = np.argsort(self.index, kind="stable")
        start = np.zeros(self.cols + 1, dtype=np.int64)
        np.add.at(start, self.index.astype(np.int64) + 1, 1)
        return Csr(self.cols, self.rows, np.cumsum(start).astype(np.int32),
                   rows_of[order].astype(np.int32), self.value[order].copy())

    def multiply(self, x: np.ndarray) -> np.ndarray:
        """y = A x with each row summed left to right (sparse.cpp:72-80)."""
        out = np.zeros(self.rows, dtype=np.float64)
        prod = self.value * x[self.index]
        # np.add.reduceat sums pairwise; the oracle owns exact order. This is
        # for host-side construction (b = A x0) only.
        nonempty = np.diff(self.start) > 0
        if prod.size:
            sums = np.add.reduceat(prod, self.start[:-1][nonempty])
            out[nonempty] = sums
        return out

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.start.astype(np.int64))


@dataclass
class Model:
    """``Model`` (model.hpp:23-49) restricted to the LP fields."""

    constraints: Csr
    objective: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    col_lower: np.ndarray
    col_upper: np.ndarray
    maximize: bool = False
    objective_offset: float = 0.0
    name: str = ""


@dataclass
class StandardLp:
    """``StandardLp`` (standard_form.hpp:23-66)."""

    k: Csr
    c: np.ndarray
    q: np.ndarray
    lower: np.ndarray
    upper: np.ndarray
    num_equalities: int
    objective_scale: float = 1.0
    objective_offset: float = 0.0
    row_origin_row: Optional[np.ndarray] = None   # int32, m
    row_origin_sign: Optional[np.ndarray] = None  # float64, m
    name: str = ""

    @property
    def num_rows(self) -> int:
        return self.k.rows

    @property
    def num_cols(self) -> int:
        return self.k.cols

    def standard_objective(self, x: np.ndarray) -> float:
        s = 0.0
        for cj, xj in zip(self.c.tolist(), np.asarray(x).tolist()):
            s += cj * xj
        return s

    def model_objective(self, x: np.ndarray) -> float:
        """``StandardLp::model_objective`` (standard_form.cpp:13-15)."""
        return self.objective_scale * self.standard_objective(x) + self.objective_offset

    def with_vectors(self, c=None, q=None, lower=None, upper=None) -> "StandardLp":
        """A case of this LP: same matrix, other data."""
        return StandardLp(self.k,
                          self.c if c is None else np.asarray(c, np.float64),
                          self.q if q is None else np.asarray(q, np.float64),
                          self.lower if lower is None else np.asarray(lower, np.float64),
                          self.upper if upper is None else np.asarray(upper, np.float64),
                          self.num_equalities, self.objective_scale,
                          self.objective_offset, self.row_origin_row,
                          self.row_origin_sign, self.name)


@dataclass
class StandardFormResult:
    ok: bool
    lp: Optional[StandardLp]
    error: str = ""
    warnings: List[str] = field(default_factory=list)
    rows_from_equalities: int = 0
    rows_from_inequalities: int = 0
    rows_from_ranges: int = 0
    free_rows_dropped: int = 0


def to_standard_form(model: Model) -> StandardFormResult:
    """``to_standard_form`` (standard_form.cpp:72-165)."""
    res = StandardFormResult(ok=False, lp=None)
    a = model.constraints
    m = a.rows
    n = a.cols
    scale = -1.0 if model.maximize else 1.0
    c = scale * np.asarray(model.objective, np.float64)
    eq, ineq = [], []  # (model_row, sign, rhs)
    for i in range(m):
        lo = float(model.row_lower[i])
        hi = float(model.row_upper[i])
        has_lo = lo > -INF
        has_hi = hi < INF
        if has_lo and has_hi and lo == hi:
            eq.append((i, 1.0, lo))
            res.rows_from_equalities += 1
        elif has_lo and has_hi:
            ineq.append((i, 1.0, lo))
            ineq.append((i, -1.0, -hi))
            res.rows_from_ranges += 1
        elif has_lo:
            ineq.append((i, 1.0, lo))
            res.rows_from_inequalities += 1
        elif has_hi:
            ineq.append((i, -1.0, -hi))
            res.rows_from_inequalities += 1
        else:
            res.free_rows_dropped += 1
    emits = eq + ineq
    mm = len(emits)
    q = np.array([e[2] for e in emits], dtype=np.float64)
    origin_row = np.array([e[0] for e in emits], dtype=np.int32)
    origin_sign = np.array([e[1] for e in emits], dtype=np.float64)
    rr, cc, vv = [], [], []
    start = a.start.astype(np.int64)
    for dest, (row, sign, _) in enumerate(emits):
        lo, hi = start[row], start[row + 1]
        rr.append(np.full(hi - lo, dest, dtype=np.int64))
        cc.append(a.index[lo:hi].astype(np.int64))
        vv.append(sign * a.value[lo:hi])
    if rr:
        k = Csr.from_triplets(mm, n, np.concatenate(rr), np.concatenate(cc),
                              np.concatenate(vv))
    else:
        k = Csr.from_triplets(mm, n, [], [], [])
    if res.free_rows_dropped > 0:
        res.warnings.append(f"{res.free_rows_dropped} row(s) with no finite bound "
                            "dropped: they constrain nothing")
    lp = StandardLp(k, c, q, np.asarray(model.col_lower, np.float64).copy(),
                    np.asarray(model.col_upper, np.float64).copy(), len(eq), scale,
                    float(model.objective_offset), origin_row, origin_sign, model.name)
    err = validate(lp)
    if err:
        res.error = "standard form failed validation: " + err
        return res
    res.ok = True
    res.lp = lp
    return res


def validate(lp: StandardLp) -> str:
    """``StandardLp::validate`` (standard_form.cpp:44-70); '' when valid."""
    k = lp.k
    if k.start.shape[0] != k.rows + 1 or k.start[0] != 0 or k.start[-1] != k.nnz:
        return "bad row starts"
    if np.any(np.diff(k.start.astype(np.int64)) < 0):
        return "start is not monotone"
    if k.nnz and (k.index.min() < 0 or k.index.max() >= k.cols):
        return "column index out of range"
    if lp.c.shape[0] != k.cols:
        return "objective length does not match columns"
    if lp.q.shape[0] != k.rows:
        return "rhs length does not match rows"
    if lp.lower.shape[0] != k.cols or lp.upper.shape[0] != k.cols:
        return "bound length does not match columns"
    if not (0 <= lp.num_equalities <= k.rows):
        return "num_equalities is out of range"
    if np.any(lp.lower > lp.upper):
        return "empty bound interval"
    if not np.all(np.isfinite(lp.q)):
        return "rhs is not finite"
    return ""
