"""The locality relabelling (anu_locality_relabel, the order
options.locality_order applies), computed on the host, against its stated
rule:

- row_old and col_old are permutations;
- the first num_equalities rows stay the equalities (the dual cone's split);
- within each block rows go by decreasing length, ties in original order;
- columns go by the first relabelled row they appear in, ties in original
  order, empty columns last.
"""
import numpy as np
import pytest

import lp_cases
from anukulan_b200 import lpgen, pdhg


def check(lp):
    row_old, col_old = pdhg.locality_relabel(lp)
    m, n, ne = lp.num_rows, lp.num_cols, lp.num_equalities
    start = np.asarray(lp.k.start)
    index = np.asarray(lp.k.index)
    assert np.array_equal(np.sort(row_old), np.arange(m))
    assert np.array_equal(np.sort(col_old), np.arange(n))
    assert set(row_old[:ne].tolist()) == set(range(ne))
    lengths = np.diff(start)
    for lo, hi in ((0, ne), (ne, m)):
        block = row_old[lo:hi]
        ln = lengths[block]
        assert np.all(np.diff(ln) <= 0)
        for v in np.unique(ln):
            assert np.all(np.diff(block[ln == v]) > 0)
    row_new = np.empty(m, np.int64)
    row_new[row_old] = np.arange(m)
    key = np.full(n, m, np.int64)
    rows_of = np.repeat(np.arange(m), lengths)
    np.minimum.at(key, index, row_new[rows_of])
    k = key[col_old]
    assert np.all(np.diff(k) >= 0)
    for v in np.unique(k):
        assert np.all(np.diff(col_old[k == v]) > 0)


def test_relabel_refinery_blocks():
    lp = lpgen.refinery_stack().base
    assert 0 < lp.num_equalities < lp.num_rows
    check(lp)


def test_relabel_power_law():
    lp, _ = lpgen.power_law_lp()
    check(lp)


@pytest.mark.parametrize("name", sorted(lp_cases.KNOWN))
def test_relabel_small(name):
    check(lp_cases.standard(lp_cases.KNOWN[name][0]()))
