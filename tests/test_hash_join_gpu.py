"""Hash join (join_algo HASH) and partitioned hash join (join_algo PARTITION)
against the CPU oracle's pair multiset: primary-key / foreign-key joins,
duplicate keys on both sides, a hot build key that overflows one
partition's shared-memory table (taken in chunks), float keys where -0.0
equals +0.0, sizes that need two radix passes, wide payloads and empty
sides.  Pairs are compared after sorting by (left row, right row)."""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import to_dev

pytestmark = pytest.mark.gpu

ALGOS = [gx.JOIN_HASH, gx.JOIN_PARTITION]


def rowid_pairs(lk, rk, algo, **kw):
    t = gx.inner_eq_join_rowids(to_dev(lk), to_dev(rk), gx.make_join_hint(algo, gx.MAT_GFUR, **kw))
    l, r = t.numpy_columns()
    o = np.lexsort((r, l))
    return l[o], r[o]


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("kdt", [np.int32, np.int64, np.uint32, np.uint64])
def test_pkfk_rowids(algo, kdt):
    npk, nfk = 1 << 15, 1 << 18
    pk = O.gen_perm(npk, kdt, seed=42)
    fk = O.gen_keys(nfk, kdt, groups=npk, seed=98, miss_frac=0.1)
    l, r = rowid_pairs(pk, fk, algo)
    el, er = O.join_pairs(pk, fk)
    assert np.array_equal(l, el) and np.array_equal(r, er)


@pytest.mark.parametrize("algo", ALGOS)
def test_left_larger_than_right(algo):
    # The smaller side builds; output columns stay in left / right order.
    lk = O.gen_keys(100_000, np.int32, groups=5000, seed=1)
    rk = O.gen_keys(7000, np.int32, groups=6000, seed=2)
    l, r = rowid_pairs(lk, rk, algo)
    el, er = O.join_pairs(lk, rk)
    assert np.array_equal(l, el) and np.array_equal(r, er)


@pytest.mark.parametrize("algo", ALGOS)
def test_hot_build_key_and_duplicates(algo):
    # 6000 build rows share one key (more than a 2048-row shared-table chunk),
    # the rest are random duplicates; every probe row of the hot key matches
    # all 6000.
    rng = np.random.default_rng(3)
    bk = rng.integers(0, 3000, size=20_000).astype(np.int64)
    bk[rng.choice(20_000, 6000, replace=False)] = 77
    pk = rng.integers(0, 4000, size=5_000).astype(np.int64)
    pk[:40] = 77
    l, r = rowid_pairs(bk, pk, algo)
    el, er = O.join_pairs(bk, pk)
    assert np.array_equal(l, el) and np.array_equal(r, er)
    assert len(l) > 40 * 6000


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("kdt", [np.float32, np.float64])
def test_float_keys_signed_zero(algo, kdt):
    rng = np.random.default_rng(4)
    lk = rng.integers(-50, 50, size=4000).astype(kdt)
    rk = rng.integers(-50, 50, size=9000).astype(kdt)
    lk[:10] = -0.0
    rk[:10] = 0.0
    l, r = rowid_pairs(lk, rk, algo)
    el, er = O.join_pairs(lk, rk)
    assert np.array_equal(l, el) and np.array_equal(r, er)


@pytest.mark.parametrize("algo", ALGOS)
def test_two_pass_partition_sizes(algo):
    # 2^21 build keys: the partitioned plan uses 11 radix bits (two passes).
    nb, npr = 1 << 21, 1 << 22
    bk = O.gen_perm(nb, np.int32, seed=5) * 3
    pk = O.gen_keys(npr, np.int32, groups=nb, seed=6, miss_frac=0.2) * 3
    m = O.join_probe_unique(bk, pk)
    l, r = rowid_pairs(bk, pk, algo)
    o = np.argsort(r, kind="stable")
    hit = np.nonzero(m >= 0)[0]
    assert np.array_equal(r[o], hit) and np.array_equal(l[o], m[hit])


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("mat", [gx.MAT_GFUR, gx.MAT_GFTR])
def test_wide_payloads(algo, mat):
    a = O.gen_keys(3000, np.int64, groups=500, seed=3)
    b = O.gen_keys(2000, np.int64, groups=700, seed=4)
    ap1 = O.gen_values(3000, np.int32, lo=0, hi=1 << 30, seed=5)
    ap2 = O.gen_values(3000, np.float64, seed=6)
    bp1 = O.gen_values(2000, np.int16, lo=-1000, hi=1000, seed=7)
    t = gx.inner_eq_join([to_dev(a), to_dev(ap1), to_dev(ap2)], [to_dev(b), to_dev(bp1)],
                         gx.make_join_hint(algo, mat))
    key, c1, c2, c3 = t.numpy_columns()
    el, er = O.join_pairs(a, b)
    exp = np.stack([a[el], ap1[el].astype(np.int64), ap2[el].view(np.int64), bp1[er].astype(np.int64)])
    got = np.stack([key, c1.astype(np.int64), c2.view(np.int64), c3.astype(np.int64)])
    assert np.array_equal(got[:, np.lexsort(got[::-1])], exp[:, np.lexsort(exp[::-1])])


@pytest.mark.parametrize("algo", ALGOS)
def test_empty_and_disjoint_sides(algo):
    e = np.zeros(0, dtype=np.int32)
    x = np.array([1, 2, 3], dtype=np.int32)
    for lk, rk in ((e, x), (x, e), (x, np.array([4, 5], np.int32))):
        t = gx.inner_eq_join_rowids(to_dev(lk), to_dev(rk), gx.make_join_hint(algo, gx.MAT_GFUR))
        assert t.num_rows == 0 and t.num_columns == 2


@pytest.mark.parametrize("algo", ALGOS)
def test_max_out_is_enforced(algo):
    x = np.arange(100, dtype=np.int32)
    with pytest.raises(gx.GxError):
        gx.inner_eq_join([to_dev(x), to_dev(x)], [to_dev(x), to_dev(x)], gx.make_join_hint(algo, gx.MAT_GFUR, max_out=50))
