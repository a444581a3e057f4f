"""Filter: predicate -> BOOL8 mask, mask -> compaction, the fused select,
and count_nonzero, against numpy on the same inputs (exact: masks,
kept rows and their order)."""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import to_dev

pytestmark = pytest.mark.gpu


def np_cmp(x, op, lo, hi):
    return {gx.CMP_LT: x < lo, gx.CMP_LE: x <= lo, gx.CMP_GT: x > lo, gx.CMP_GE: x >= lo, gx.CMP_EQ: x == lo,
            gx.CMP_NE: x != lo, gx.CMP_BETWEEN: (x >= lo) & (x < hi)}[op]


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 1 << 20])
def test_date_range_select_like_the_batched_pipeline(n):
    # The batched workload's filter: lo <= date < hi on an int32 date column.
    date = O.gen_values(n, np.int32, lo=0, hi=2557, seed=1)
    amount = O.gen_values(n, np.int64, lo=100, hi=10**7, seed=2)
    code = O.gen_values(n, np.int32, lo=0, hi=10**4, seed=3)
    cols = [to_dev(date), to_dev(amount), to_dev(code)]
    p = [gx.predicate(0, gx.CMP_BETWEEN, 500, 500 + 1023)]
    keep = (date >= 500) & (date < 1523)
    m = gx.select_to_bitmask(cols, p).cpu().numpy()
    assert np.array_equal(m.astype(bool), keep)
    t = gx.select(cols, p)
    d, a, c = t.numpy_columns()
    assert np.array_equal(d, date[keep]) and np.array_equal(a, amount[keep]) and np.array_equal(c, code[keep])
    t2 = gx.compact(cols, to_dev(keep.astype(np.uint8)).view(__import__("torch").bool))
    for x, y in zip(t2.numpy_columns(), (date[keep], amount[keep], code[keep])):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("combine", [gx.COMBINE_AND, gx.COMBINE_OR])
def test_every_comparison_on_every_type(combine):
    n = 100_003
    rng = np.random.default_rng(4)
    cols = {
        np.int8: rng.integers(-100, 100, n).astype(np.int8),
        np.uint16: rng.integers(0, 60000, n).astype(np.uint16),
        np.int32: rng.integers(-10**6, 10**6, n).astype(np.int32),
        np.uint64: rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2),
        np.float32: rng.normal(size=n).astype(np.float32),
        np.float64: rng.normal(size=n),
    }
    arrs = list(cols.values())
    lits = [(-3, 40), (1000, 50000), (-5000, 123456), (2**63 + 5, 2**64 - 10), (-0.25, 0.5), (0.1, 1.5)]
    for op in range(7):
        preds = []
        expect = np.ones(n, bool) if combine == gx.COMBINE_AND else np.zeros(n, bool)
        for j, (a, (lo, hi)) in enumerate(zip(arrs, lits)):
            preds.append(gx.predicate(j, op, lo, hi))
            e = np_cmp(a, op, a.dtype.type(lo), a.dtype.type(hi))
            expect = expect & e if combine == gx.COMBINE_AND else expect | e
        m = gx.select_to_bitmask([to_dev(a) for a in arrs], preds, combine).cpu().numpy().astype(bool)
        assert np.array_equal(m, expect), op
        t = gx.select([to_dev(a) for a in arrs], preds, combine)
        for got, a in zip(t.numpy_columns(), arrs):
            assert np.array_equal(got, a[expect])


def test_count_nonzero_and_validation():
    v = np.array([0, 1, -1, 0, 5], np.int64)
    assert gx.count_nonzero(to_dev(v)) == 3
    f = np.array([0.0, -0.0, np.nan, 2.0], np.float64)
    assert gx.count_nonzero(to_dev(f)) == 2  # NaN != 0, -0.0 == 0
    x = to_dev(np.arange(10, dtype=np.int32))
    with pytest.raises(gx.GxError):
        gx.select([x], [gx.predicate(3, gx.CMP_LT, 1)])  # column out of range
    with pytest.raises(gx.GxError):
        gx.select([x], [])  # no predicate
