"""The CPU oracle checked against the reference's own tests (no GPU).

* tests/golden/groupby_multikeys.json — the literal cases of the reference's
  src/cuda/tests/groupby/groupby_multikeys_test.cu (extracted by
  tests/golden/make_golden.py).  Multi-column keys are fused into one int64
  key per distinct tuple, the way the reference's smart key fusion feeds a
  single-key group-by.
* The closed forms of src/cuda/tests/groupby/groupby_test.hpp:64-92,
  the PK-FK counts of src/cuda/tests/join/ieq_join_test.cu:19-83, the
  dictionary properties of src/cuda/tests/compress/dictionary_encode_test.cu
  and the partition checks of src/cuda/tests/sort/sort_partition_test.cu.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O

GOLD = Path(__file__).resolve().parent / "golden" / "groupby_multikeys.json"
KIND = {"SUM": O.SUM, "MAX": O.MAX, "MIN": O.MIN, "AVG": O.AVG, "ANY": O.ANY, "COUNT_ALL": O.COUNT_ALL}
TYPES = {"INT64": np.int64, "FLOAT64": np.float64, "INT32": np.int32, "FLOAT32": np.float32}


def _cases():
    doc = json.loads(GOLD.read_text())
    return [c for c in doc["cases"] if c["ok"] and c["expects"]]


def fuse_keys(cols: list[np.ndarray]) -> tuple[np.ndarray, dict]:
    """One int64 id per distinct key tuple (an injective key fusion)."""
    tuples = list(zip(*[c.tolist() for c in cols]))
    ids = {t: i for i, t in enumerate(sorted(set(tuples)))}
    return np.array([ids[t] for t in tuples], dtype=np.int64), ids


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference_multikey_vectors(case):
    keys = [np.array(k["values"], dtype=k["dtype"]) for k in case["keys"]]
    vals = [np.array(v["values"], dtype=v["dtype"]) for v in case["vals"]]
    fused, ids = fuse_keys(keys)
    reqs = [(c, KIND[k]) for c, k in case["requests"]]
    out = O.groupby(fused, vals, reqs, agg_count=case["agg_count"])
    nkeys = len(keys)
    if case["num_rows"] is not None:
        assert len(out[0]) == case["num_rows"]
    if case["num_columns"] is not None:
        assert nkeys + len(out) - 1 == case["num_columns"]
    for col, tname in case["column_types"].items():
        assert out[int(col) - nkeys + 1].dtype == TYPES[tname]
    inv = {v: k for k, v in ids.items()}
    for e in case["expects"]:
        c = e["column"]
        if "row" in e:
            row = e["row"]
        else:
            row = int(np.nonzero(out[0] == ids[tuple(e["key"])])[0][0])
        if c < nkeys:
            got = inv[int(out[0][row])][c]
        else:
            got = out[c - nkeys + 1][row]
        if e["tol"]:
            assert abs(float(got) - e["value"]) <= e["tol"], (case["name"], e, got)
        else:
            assert got == e["value"], (case["name"], e, got)


@pytest.mark.parametrize("G", [4, 32, 1024, 1 << 14])
def test_uniform_closed_form(G):
    # groupby_test.hpp:64-74: keys i % G shuffled, all-ones values: every
    # group sums to N/G and the keys sum to G(G-1)/2.
    n = 1 << 16
    k = O.gen_keys(n, np.int32, dist=O.DIST_CYCLIC, groups=G, seed=7)
    ones = np.ones(n, dtype=np.int32)
    out = O.groupby(k, [ones, ones], [(0, O.SUM), (1, O.SUM)])
    assert len(out[0]) == G
    assert np.all(out[1] == n // G) and np.all(out[2] == n // G)
    assert int(out[0].astype(np.int64).sum()) == G * (G - 1) // 2


@pytest.mark.parametrize("s", [0.5, 1.0, 2.0])
def test_zipf_closed_form(s):
    # groupby_test.hpp:81-92: each group's sum of ones equals the key's count.
    n, G = 1 << 16, 1024
    k = O.gen_keys(n, np.int32, dist=O.DIST_ZIPF, groups=G, zipf_s=s, seed=3)
    out = O.groupby(k, [np.ones(n, np.int32)], [(0, O.SUM)])
    counts = np.bincount(k, minlength=G)
    assert np.array_equal(out[1], counts[out[0]])
    assert len(out[0]) == np.count_nonzero(counts)


def test_groupby_int64_keys_and_all_aggregates():
    n = 5000
    k = O.gen_keys(n, np.int64, groups=97, scatter=1, seed=11)
    v = O.gen_values(n, np.int64, lo=-1000, hi=1000, seed=12)
    f = O.gen_values(n, np.float64, seed=13)
    out = O.groupby(k, [v, f], [(0, O.SUM), (0, O.MIN), (0, O.MAX), (1, O.SUM), (1, O.MIN), (1, O.MAX),
                                (1, O.AVG), (0, O.COUNT_ALL)])
    for i, key in enumerate(out[0]):
        m = k == key
        assert out[1][i] == v[m].sum() and out[2][i] == v[m].min() and out[3][i] == v[m].max()
        assert abs(out[4][i] - f[m].sum()) <= 1e-12 * abs(f[m].sum())
        assert out[5][i] == f[m].min() and out[6][i] == f[m].max()
        assert abs(out[7][i] - f[m].mean()) <= 1e-12
        assert out[8][i] == m.sum()
    assert np.all(np.diff(out[0]) > 0)


def test_join_pkfk_counts():
    # ieq_join_test.cu:47-83: PK side = permutation of 0..npk-1, FK side
    # uniform over the PK keys -> one match per FK row.
    npk, nfk = 1024, 4096
    pk = O.gen_perm(npk, np.int32, seed=42)
    fk = O.gen_keys(nfk, np.int32, groups=npk, seed=98)
    l, r = O.join_pairs(pk, fk)
    assert len(l) == nfk
    assert np.array_equal(pk[l], fk[r])
    # 10% absent keys -> only the present ones match.
    fk2 = O.gen_keys(nfk, np.int32, groups=npk, seed=5, miss_frac=0.1)
    l2, r2 = O.join_pairs(pk, fk2)
    assert len(l2) == int(np.sum(fk2 < npk))
    assert O.join_count_parallel(pk, fk2) == len(l2)


def test_join_many_to_many():
    a = np.array([1, 1, 2, 3, 3, 3], dtype=np.int64)
    b = np.array([3, 1, 4, 3], dtype=np.int64)
    l, r = O.join_pairs(a, b)
    exp = sorted((i, j) for i in range(len(a)) for j in range(len(b)) if a[i] == b[j])
    assert list(zip(l.tolist(), r.tolist())) == exp


def test_dictionary_properties():
    # dictionary_encode_test.cu:16-52 (bijection, NDV, dense) and 160-202 (rank).
    k = O.gen_keys(4096, np.int32, groups=256, scatter=1, seed=1)
    codes, nd = O.dict_encode(k)
    assert nd == len(np.unique(k))
    assert set(codes.tolist()) == set(range(nd))
    pairs = set(zip(k.tolist(), codes.tolist()))
    assert len(pairs) == nd
    rcodes, nd2 = O.dict_encode(k, ordered=True)
    uniq = np.unique(k)
    assert nd2 == nd and np.array_equal(rcodes, np.searchsorted(uniq, k))
    d = O.gen_perm(64, np.int32, seed=4)
    q = np.concatenate([d[::3], np.array([1000, -5], dtype=np.int32)])
    pos = O.dict_with_dict(q, d)
    assert np.array_equal(pos[:-2], np.arange(0, 64, 3)) and np.all(pos[-2:] == np.iinfo(np.int32).min)


@pytest.mark.parametrize("dtype", [np.int32, np.int64])
def test_partition_permutation(dtype):
    # sort_partition_test.cu:16-42: partition on bits 0..5 keeps (key, val)
    # aligned and is a permutation; offsets are inclusive.
    n = 4864
    k = O.gen_keys(n, dtype, groups=2 * n, seed=42)
    v = np.arange(n, dtype=np.int64)
    pk, pv = O.sort_pairs(k, v, 0, 5)
    assert np.array_equal(np.sort(pv), v) and np.array_equal(k[pv], pk)
    d = pk.astype(np.int64) & 31
    assert np.all(np.diff(d) >= 0)
    # stable within a partition
    for p in range(32):
        idx = pv[d == p]
        assert np.all(np.diff(idx) > 0)
    off = O.partition_offsets(pk, 0, 5)
    assert off[-1] == n and np.array_equal(off[:-1], np.cumsum(np.bincount(d, minlength=32)))


def test_sort_signed_float_and_descending():
    k = np.array([3, -1, 0, -7, 5, -1, 2], dtype=np.int32)
    sk, idx = O.sort_pairs(k, iota=True)
    assert np.array_equal(sk, np.sort(k, kind="stable")) and np.array_equal(idx, np.argsort(k, kind="stable"))
    f = np.array([0.5, -0.0, 0.0, -2.5, np.inf, -np.inf, 1e-300], dtype=np.float64)
    sf, fi = O.sort_pairs(f, iota=True)
    assert np.array_equal(sf[[0, 1]], [-np.inf, -2.5]) and sf[-1] == np.inf
    assert set(fi[2:4].tolist()) == {1, 2}  # -0.0 and +0.0 tie, stable
    sd, di = O.sort_pairs(k, iota=True, desc=True)
    assert np.array_equal(sd, -np.sort(-k, kind="stable")) and di[0] == 4


def test_generators_cyclic_exact_and_hll():
    k = O.gen_keys(1 << 14, np.int64, dist=O.DIST_CYCLIC, groups=100, seed=9)
    c = np.bincount(k)
    assert c.max() - c.min() <= 1
    big = O.gen_keys(1 << 20, np.int64, groups=1 << 18, scatter=1, seed=2)
    est = O.hll_estimate(O.hll_registers(big))
    exact = O.ndv_exact(big)
    assert abs(est - exact) / exact < 0.04


@pytest.mark.parametrize("vdt", [np.int8, np.int16, np.int32, np.uint32, np.int64, np.uint64, np.float32, np.float64])
def test_groupby_value_types_against_numpy(vdt):
    # Output types follow the reference (agg_func.cuh:20-60): integer SUM
    # widens to 64 bits (signedness kept), float SUM keeps the float type
    # (accumulated in higher precision, rounded once), MIN/MAX keep the input
    # type, AVG is double, COUNT int64.
    n = 4000
    k = O.gen_keys(n, np.int32, groups=37, scatter=1, seed=21)
    if np.dtype(vdt).kind == "f":
        v = ((O.gen_values(n, np.float64, seed=22) - 0.5) * 100).astype(vdt)
    else:
        info = np.iinfo(vdt)
        v = O.gen_values(n, np.int64, lo=max(int(info.min), -(1 << 30)), hi=min(int(info.max), 1 << 30),
                         seed=22).astype(vdt)
    out = O.groupby(k, [v], [(0, O.SUM), (0, O.MIN), (0, O.MAX), (0, O.AVG), (0, O.COUNT_ALL)])
    for i, key in enumerate(out[0]):
        m = k == key
        x = v[m]
        if np.dtype(vdt).kind == "f":
            rtol = 1e-6 if vdt == np.float32 else 1e-12
            ref = x.astype(np.float64).sum()
            assert out[1].dtype == vdt
            assert abs(float(out[1][i]) - ref) <= rtol * max(1.0, abs(ref))
        else:
            assert int(out[1][i]) == int(x.astype(np.int64 if np.dtype(vdt).kind == "i" else np.uint64).sum())
        assert out[2][i] == x.min() and out[3][i] == x.max()
        assert out[2].dtype == vdt and out[3].dtype == vdt
        assert abs(out[4][i] - x.astype(np.float64).mean()) <= 1e-9 * max(1.0, abs(x.astype(np.float64).mean()))
        assert out[5][i] == m.sum()


def test_groupby_float_nan_semantics():
    # NaN takes part in SUM (the sum becomes NaN) but not in MIN/MAX; a group
    # of NaNs only keeps the identities.
    k = np.array([1, 1, 1, 2, 2, 3], dtype=np.int32)
    v = np.array([1.5, np.nan, -2.0, np.nan, np.nan, 4.0], dtype=np.float64)
    out = O.groupby(k, [v], [(0, O.SUM), (0, O.MIN), (0, O.MAX), (0, O.COUNT_ALL)])
    assert list(out[0]) == [1, 2, 3]
    assert np.isnan(out[1][0]) and np.isnan(out[1][1]) and out[1][2] == 4.0
    assert out[2][0] == -2.0 and out[3][0] == 1.5
    assert out[2][2] == 4.0 and out[3][2] == 4.0
    assert list(out[4]) == [3, 2, 1]
