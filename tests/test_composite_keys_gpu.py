"""Group-by and distinct on STRING keys and on several key columns (with
and without smart key fusion), the fused key itself, and gather of numeric
and STRING columns — through the C ABI, against the CPU oracle.

Expected results: the key rows are numbered on the CPU (np.unique over the
key tuples), the oracle groups the values by that number, and each group's
key tuple is attached; both sides are then compared as key -> aggregate
maps (integers exact, float64 SUM within 1e-12 relative)."""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import FLOAT_RTOL, to_dev

pytestmark = pytest.mark.gpu

REQS = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MAX), (0, gx.COUNT_ALL)]
OREQS = [(0, O.SUM), (0, O.MIN), (0, O.MAX), (1, O.SUM), (1, O.MAX), (0, O.COUNT_ALL)]


def vocab(n, seed, max_len=40):
    rng = np.random.default_rng(seed)
    words = set()
    while len(words) < n:
        ln = int(rng.integers(0, max_len + 1))
        words.add(bytes(rng.integers(32, 127, size=ln, dtype=np.uint8)))
    return sorted(words)


def expected(key_cols, vals):
    """key tuple -> (aggregates...) from the oracle over CPU-numbered groups."""
    n = len(key_cols[0])
    rows = list(zip(*[list(c) for c in key_cols])) if n else []
    index = {}
    ids = np.empty(n, dtype=np.int64)
    for i, r in enumerate(rows):
        ids[i] = index.setdefault(r, len(index))
    out = O.groupby(ids, vals, OREQS)
    keys = {g: r for r, g in index.items()}
    return {keys[int(g)]: tuple(c[j] for c in out[1:]) for j, g in enumerate(out[0])}


def got_map(t, nkeys):
    cols = t.numpy_columns()
    res = {}
    for j in range(t.num_rows):
        k = tuple(c[j].item() if isinstance(c[j], np.generic) else c[j] for c in cols[:nkeys])
        assert k not in res, f"key {k} emitted twice"
        res[k] = tuple(c[j] for c in cols[nkeys:])
    return res


def assert_maps_equal(got, exp):
    assert set(got) == set(exp)
    for k, e in exp.items():
        g = got[k]
        for a, b in zip(g, e):
            if isinstance(b, (float, np.floating)):
                assert abs(a - b) <= FLOAT_RTOL * max(abs(b), 1e-300), (k, a, b)
            else:
                assert a == b, (k, a, b)


def norm(col):
    """Numpy key column -> python values comparable with the table's."""
    return [x.item() if isinstance(x, np.generic) else x for x in col]


@pytest.mark.parametrize("algo", [gx.HASH, gx.SORT, gx.AUTO_ALGO])
def test_string_key_groupby(algo):
    n = 100_000
    words = vocab(700, 1)
    rng = np.random.default_rng(2)
    kid = rng.integers(0, len(words), size=n)
    keys = [words[i] for i in kid]
    iv = O.gen_values(n, np.int64, lo=-1000, hi=10**9, seed=3)
    fv = O.gen_values(n, np.float64, seed=4)
    hint = gx.make_hint(algo)
    t = gx.groupby([gx.StringColumn.from_list(keys)], [to_dev(iv), to_dev(fv)], REQS, hint)
    assert hint.groupby_algo in (gx.HASH, gx.SORT)
    assert_maps_equal(got_map(t, 1), expected([keys], [iv, fv]))


def test_string_key_with_row_offset_and_empty_strings():
    words = [b"", b"a", b"ab", b"a" * 100, b"\x00\x01", b"zz"]
    rng = np.random.default_rng(5)
    keys = [words[i] for i in rng.integers(0, len(words), size=5000)]
    sc = gx.StringColumn.from_list(keys)
    view = gx.StringColumn(sc.chars, sc.offsets, rows=4000, row_offset=1000)
    iv = O.gen_values(4000, np.int64, lo=0, hi=100, seed=6)
    t = gx.groupby([view], [to_dev(iv)], [(0, gx.SUM), (0, gx.COUNT_ALL)], gx.make_hint(gx.HASH))
    exp = O.groupby(np.array([words.index(k) for k in keys[1000:]], np.int64), [iv], [(0, O.SUM), (0, O.COUNT_ALL)])
    e = {words[int(g)]: (s, c) for g, s, c in zip(*exp)}
    g = {k: (s, c) for k, s, c in zip(*t.numpy_columns())}
    assert g == e


def test_string_key_partition_is_rejected_like_the_reference():
    sc = gx.StringColumn.from_list([b"a", b"b"])
    with pytest.raises(gx.GxError, match="STRING keys not supported"):
        gx.groupby([sc], [to_dev(np.arange(2, dtype=np.int64))], [(0, gx.SUM)], gx.make_hint(gx.PARTITION))


@pytest.mark.parametrize("skf", [0, 1])
@pytest.mark.parametrize("algo", [gx.HASH, gx.SORT])
def test_multi_column_integer_keys(skf, algo):
    n = 200_000
    rng = np.random.default_rng(7)
    a = rng.integers(-50, 50, size=n).astype(np.int32)
    b = rng.integers(0, 2**40, size=60, dtype=np.int64)[rng.integers(0, 60, size=n)]  # wide range, 60 values
    c = rng.integers(0, 4, size=n).astype(np.uint8)
    iv = O.gen_values(n, np.int64, lo=0, hi=1 << 31, seed=8)
    fv = O.gen_values(n, np.float64, seed=9)
    hint = gx.make_hint(algo, enable_skf=skf)
    t = gx.groupby([to_dev(a), to_dev(b), to_dev(c)], [to_dev(iv), to_dev(fv)], REQS, hint)
    assert t.num_columns == 3 + len(REQS)
    assert_maps_equal(got_map(t, 3), expected([norm(a), norm(b), norm(c)], [iv, fv]))


def test_skf_allows_partition_and_agg_count():
    n = 100_000
    rng = np.random.default_rng(10)
    a = rng.integers(0, 300, size=n).astype(np.int64)
    b = rng.integers(-8, 8, size=n).astype(np.int16)
    iv = O.gen_values(n, np.int64, lo=0, hi=1000, seed=11)
    hint = gx.make_hint(gx.PARTITION, enable_skf=1, agg_count=1)
    t = gx.groupby([to_dev(a), to_dev(b)], [to_dev(iv)], [(0, gx.SUM)], hint)
    cols = t.numpy_columns()
    assert len(cols) == 4  # a, b, SUM, trailing COUNT
    exp = expected([norm(a), norm(b)], [iv, iv])
    g = {(x.item(), y.item()): (s, c) for x, y, s, c in zip(*cols)}
    assert g == {k: (v[0], v[5]) for k, v in exp.items()}


def test_multi_column_keys_without_skf_reject_partition():
    x = to_dev(np.arange(10, dtype=np.int32))
    with pytest.raises(gx.GxError, match="single-column"):
        gx.groupby([x, x], [x], [(0, gx.SUM)], gx.make_hint(gx.PARTITION))


@pytest.mark.parametrize("skf", [0, 1])
def test_mixed_string_float_int_keys(skf):
    # STRING and float columns cannot be bit-packed: SKF falls back to the
    # chained dictionary codes; -0.0 and +0.0 are one key.
    n = 60_000
    rng = np.random.default_rng(12)
    words = vocab(40, 13, max_len=12)
    s = [words[i] for i in rng.integers(0, len(words), size=n)]
    f = rng.integers(-3, 4, size=n).astype(np.float64)
    f[f == 0] = np.where(rng.random(int((f == 0).sum())) < 0.5, -0.0, 0.0)
    i = rng.integers(0, 5, size=n).astype(np.int64)
    iv = O.gen_values(n, np.int64, lo=0, hi=1 << 20, seed=14)
    fv = O.gen_values(n, np.float64, seed=15)
    t = gx.groupby([gx.StringColumn.from_list(s), to_dev(f), to_dev(i)], [to_dev(iv), to_dev(fv)], REQS,
                   gx.make_hint(gx.HASH, enable_skf=skf))
    exp = expected([s, [x + 0.0 for x in norm(f)], norm(i)], [iv, fv])
    got = {(k[0], k[1] + 0.0, k[2]): v for k, v in got_map(t, 3).items()}
    assert_maps_equal(got, exp)


@pytest.mark.parametrize("algo", [gx.HASH, gx.SORT])
def test_distinct_string_and_multi_column(algo):
    rng = np.random.default_rng(16)
    words = vocab(300, 17)
    s = [words[i] for i in rng.integers(0, len(words), size=50_000)]
    t = gx.distinct([gx.StringColumn.from_list(s)], algo=algo)
    got = list(t.to_numpy(0))
    assert sorted(got) == sorted(set(s)) and len(got) == len(set(s))
    a = rng.integers(0, 30, size=50_000).astype(np.int32)
    b = rng.integers(0, 30, size=50_000).astype(np.int64)
    t = gx.distinct([to_dev(a), to_dev(b)], algo=algo)
    ga, gb = t.numpy_columns()
    assert sorted(zip(ga.tolist(), gb.tolist())) == sorted(set(zip(a.tolist(), b.tolist())))


def test_empty_composite_inputs():
    e32, e64 = np.zeros(0, np.int32), np.zeros(0, np.int64)
    t = gx.groupby([to_dev(e32), to_dev(e64)], [to_dev(e64)], [(0, gx.SUM)], gx.make_hint(gx.HASH))
    assert t.num_rows == 0 and t.num_columns == 3
    t = gx.distinct([gx.StringColumn.from_list([])])
    assert t.num_rows == 0


def test_multikey_compress_equality_and_bits():
    n = 50_000
    rng = np.random.default_rng(18)
    a = rng.integers(-5, 3, size=n).astype(np.int32)   # range 7: 3 bits
    b = rng.integers(100, 164, size=n).astype(np.uint16)  # range <= 63: 6 bits
    fused, bits = gx.multikey_compress([to_dev(a), to_dev(b)])
    assert bits == 3 + 6
    f = fused.cpu().numpy().view(np.uint64)
    pairs = a.astype(np.int64) * 1000 + b
    # equal fused keys <=> equal key rows: fused key <-> key row is a bijection
    both = set(zip(f.tolist(), pairs.tolist()))
    assert len(both) == len(set(f.tolist())) == len(set(pairs.tolist()))
    assert gx.multikey_compress([to_dev(a), to_dev(np.zeros(n, np.float32))]) is None
    # Wide-range columns fall back to dictionary codes: 50000 distinct values
    # take 16 bits each.
    wide = rng.integers(-2**62, 2**62, size=n, dtype=np.int64)
    fused, bits = gx.multikey_compress([to_dev(wide), to_dev(wide[::-1].copy())])
    assert bits == 32
    f = fused.cpu().numpy().view(np.uint64)
    assert len(set(zip(f.tolist(), wide.tolist(), wide[::-1].tolist()))) == len(set(f.tolist())) == n
    # Three columns of ~2^22 distinct values need 3 x 23 bits: more than 64.
    m = 1 << 22
    cols = [to_dev(rng.integers(-2**62, 2**62, size=m, dtype=np.int64)) for _ in range(3)]
    assert gx.multikey_compress(cols, max_bits=64) is None


def test_gather_numeric_and_strings():
    rng = np.random.default_rng(19)
    v = rng.integers(-2**40, 2**40, size=1000, dtype=np.int64)
    idx = rng.integers(0, 1000, size=3000).astype(np.int64)
    assert np.array_equal(gx.gather(to_dev(idx), to_dev(v)).cpu().numpy(), v[idx])
    words = vocab(200, 20)
    strs = [words[i] for i in rng.integers(0, 200, size=1000)]
    got = gx.gather(to_dev(idx), gx.StringColumn.from_list(strs))
    assert list(got) == [strs[i] for i in idx]
