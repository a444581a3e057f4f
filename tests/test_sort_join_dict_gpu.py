"""Parity of the radix sort / partition, sort-based join, dictionary
encoding, HLL sketch and generators (CUDA library vs CPU oracle).
Sort, partition, partition offsets, ordered dictionary codes and HLL
registers-derived estimates are bit-exact; join pairs are bit-exact after
canonical sort; hash dictionary codes are checked as a bijection."""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import to_dev

pytestmark = pytest.mark.gpu


# ----------------------------------------------------------------- sort ----
@pytest.mark.parametrize("kdt", [np.int32, np.int64, np.uint32, np.float32, np.float64, np.int16, np.int8])
@pytest.mark.parametrize("bits", [(0, -1), (0, 5), (3, 17), (8, 16)])
@pytest.mark.parametrize("desc", [False, True])
def test_sort_pairs_bit_exact(kdt, bits, desc):
    n = 70001
    if np.dtype(kdt).kind == "f":
        k = (O.gen_values(n, np.float64, seed=1) * 2000 - 1000).astype(kdt)
        k[::97] = -0.0
    else:
        k = O.gen_keys(n, np.int64, groups=1 << 40, seed=2).astype(kdt)
    b, e = bits
    if e > 8 * np.dtype(kdt).itemsize:
        pytest.skip("bit range beyond key width")
    v = O.gen_values(n, np.int64, lo=0, hi=1 << 50, seed=3)
    sk, sv = gx.sort_column_pair(to_dev(k), to_dev(v), b, e, gx.DESCENDING if desc else gx.ASCENDING)
    ek, ev = O.sort_pairs(k, v, b, e, desc)
    assert np.array_equal(sk.cpu().numpy().view(np.uint8), ek.view(np.uint8))
    assert np.array_equal(sv.cpu().numpy(), ev)


@pytest.mark.parametrize("per_tile", [False, True])
@pytest.mark.parametrize("kdt,vdt", [(np.int32, np.int64), (np.float64, np.int32), (np.uint64, np.float64)])
def test_sort_pairs_persistent_and_per_tile_passes(monkeypatch, per_tile, kdt, vdt):
    # Several tiles per SM and a partial last tile, through the persistent
    # bulk-copy digit passes and through the per-tile kernel
    # (GX_RADIX_NO_BULK): both bit-exact, ascending and descending, on a bit
    # range and on row ids.
    if per_tile:
        monkeypatch.setenv("GX_RADIX_NO_BULK", "1")
    n = 148 * 3 * 4096 + 1234
    if np.dtype(kdt).kind == "f":
        k = (O.gen_values(n, np.float64, seed=5) * 2000 - 1000).astype(kdt)
    else:
        k = O.gen_keys(n, np.int64, groups=1 << 40, seed=6).astype(kdt)
    v = O.gen_values(n, np.int64, lo=0, hi=1 << 30, seed=7).astype(vdt)
    for b, e, desc in ((0, -1, False), (0, -1, True), (3, 21, False)):
        sk, sv = gx.sort_column_pair(to_dev(k), to_dev(v), b, e, gx.DESCENDING if desc else gx.ASCENDING)
        ek, ev = O.sort_pairs(k, v, b, e, desc)
        assert np.array_equal(sk.cpu().numpy().view(np.uint8), ek.view(np.uint8))
        assert np.array_equal(sv.cpu().numpy().view(np.uint8), ev.view(np.uint8))
    sk, idx = gx.argsort(to_dev(k))
    ek, ei = O.sort_pairs(k, iota=True)
    assert np.array_equal(sk.cpu().numpy().view(np.uint8), ek.view(np.uint8))
    assert np.array_equal(idx.cpu().numpy(), ei)


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 1 << 20])
def test_argsort_and_sort_column(n):
    k = O.gen_keys(n, np.int64, groups=1000, scatter=1, seed=4) if n else np.zeros(0, np.int64)
    sk, idx = gx.argsort(to_dev(k))
    ek, ei = O.sort_pairs(k, iota=True)
    assert np.array_equal(sk.cpu().numpy(), ek) and np.array_equal(idx.cpu().numpy(), ei)
    only = gx.sort_column(to_dev(k))
    assert np.array_equal(only.cpu().numpy(), ek)


@pytest.mark.parametrize("kdt", [np.int32, np.int64])
def test_partition_and_offsets_reference_case(kdt):
    # sort_partition_test.cu:16-59 shapes (4864 / 4865 rows, bits 0..5).
    for nrows in (4864, 4865):
        k = O.gen_keys(2 * nrows, kdt, groups=nrows, seed=42)
        v = np.arange(2 * nrows, dtype=np.int64)
        pk, pv = gx.partition_column_pair(to_dev(k), to_dev(v), 0, 5)
        ek, ev = O.sort_pairs(k, v, 0, 5)
        assert np.array_equal(pk.cpu().numpy(), ek) and np.array_equal(pv.cpu().numpy(), ev)
        off = gx.compute_partition_offsets(pk, 0, 5).cpu().numpy()
        assert np.array_equal(off, O.partition_offsets(ek, 0, 5))
        ak, ai = gx.arg_partition(to_dev(k), 0, 5)
        assert np.array_equal(ai.cpu().numpy(), ev)


def test_sort_large_property():
    import torch
    n = 1 << 26
    k = torch.empty(n, dtype=torch.int32, device="cuda")
    gx.generate_keys(k, gx.gen_spec(seed=9, groups=1 << 30, scatter=1))
    sk, idx = gx.argsort(k)
    assert bool((sk[1:] >= sk[:-1]).all())
    assert bool((k[idx] == sk).all())
    counts = torch.bincount(idx, minlength=n)
    assert bool((counts == 1).all())


# ----------------------------------------------------------------- join ----
def canon_pairs(t, rowids=True):
    cols = t.numpy_columns()
    if rowids:
        l, r = cols
    else:
        l, r = cols[1], cols[2]
    o = np.lexsort((r, l))
    return l[o], r[o]


@pytest.mark.parametrize("mode", [gx.SORTED_BUILD, gx.SORT_MERGE])
@pytest.mark.parametrize("kdt", [np.int32, np.int64])
def test_join_rowids_pkfk(mode, kdt):
    npk, nfk = 1 << 14, 1 << 17
    pk = O.gen_perm(npk, kdt, seed=42)
    fk = O.gen_keys(nfk, kdt, groups=npk, seed=98, miss_frac=0.1)
    t = gx.inner_eq_join_rowids(to_dev(pk), to_dev(fk), gx.make_join_hint(sort_mode=mode))
    l, r = canon_pairs(t)
    el, er = O.join_pairs(pk, fk)
    assert np.array_equal(l, el) and np.array_equal(r, er)


@pytest.mark.parametrize("mode", [gx.SORTED_BUILD, gx.SORT_MERGE])
@pytest.mark.parametrize("mat", [gx.MAT_GFUR, gx.MAT_GFTR])
def test_join_narrow_payload_layout(mode, mat):
    # C3 shape at reduced size: [key, left payload (row id), right payload (row id)].
    nb, npr = 1 << 12, 1 << 15
    bk = O.gen_perm(nb, np.int32, seed=1)
    pk = O.gen_keys(npr, np.int32, dist=O.DIST_ZIPF, groups=nb, zipf_s=1.0, seed=2)
    pk = bk[pk]  # skewed over the build keys
    lrow = np.arange(nb, dtype=np.int64)
    rrow = np.arange(npr, dtype=np.int64)
    hint = gx.make_join_hint(gx.JOIN_SORT, mat, sort_mode=mode, unique_left=1)
    t = gx.inner_eq_join([to_dev(bk), to_dev(lrow)], [to_dev(pk), to_dev(rrow)], hint)
    key, lp, rp = t.numpy_columns()
    o = np.lexsort((rp, lp))
    el, er = O.join_pairs(bk, pk)
    assert np.array_equal(lp[o], el) and np.array_equal(rp[o], er)
    assert np.array_equal(key[o], bk[el])


@pytest.mark.parametrize("two_pass", [False, True])
@pytest.mark.parametrize("mode", [gx.SORTED_BUILD, gx.SORT_MERGE])
@pytest.mark.parametrize("kdt", [np.int32, np.int64])
def test_join_sparse_unique_build_single_pass(monkeypatch, mode, kdt, two_pass):
    # Unique build keys spread 8 apart (too sparse for direct placement):
    # the sorted-build and sort-merge matchers probe in one pass with the
    # tiles placed by look-back (GX_JOIN_TWO_PASS: count, scan, write).
    # Several tiles, a partial last tile, 10% absent probe keys, payloads of
    # both sides and the row-id form.
    if two_pass:
        monkeypatch.setenv("GX_JOIN_TWO_PASS", "1")
    nb, npr = 5000, 3 * 4096 + 777
    bk = (O.gen_perm(nb, kdt, seed=21) * 8 - 40000).astype(kdt)
    pick = O.gen_keys(npr, np.int64, groups=nb, seed=22)
    pk = bk[pick].copy()
    pk[::10] = 3  # 3 is not a multiple of 8 away from -40000: absent
    bpay = O.gen_values(nb, np.float64, seed=23)
    ppay = O.gen_values(npr, np.int32, lo=-5, hi=5, seed=24)
    hint = gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, sort_mode=mode)
    t = gx.inner_eq_join([to_dev(bk), to_dev(bpay)], [to_dev(pk), to_dev(ppay)], hint)
    key, c1, c2 = t.numpy_columns()
    el, er = O.join_pairs(bk, pk)
    exp = np.stack([bk[el].astype(np.int64), bpay[el].view(np.int64), ppay[er].astype(np.int64)])
    got = np.stack([key.astype(np.int64), c1.view(np.int64), c2.astype(np.int64)])
    assert got.shape == exp.shape
    assert np.array_equal(got[:, np.lexsort(got[::-1])], exp[:, np.lexsort(exp[::-1])])
    r = gx.inner_eq_join_rowids(to_dev(bk), to_dev(pk), hint)
    l, p = r.numpy_columns()
    o = np.lexsort((p, l))
    assert np.array_equal(l[o], el) and np.array_equal(p[o], er)


def test_join_dense_build_with_gaps():
    # Unique build keys covering 3/4 of their range (direct placement with
    # empty positions) and, with SORTED_BUILD, the sorted-build matcher.
    # Probe keys hit, fall into gaps and fall outside the range; several
    # tiles and a partial last one.
    span = 40000
    rng = np.random.default_rng(31)
    bk = rng.permutation(span)[: span * 3 // 4].astype(np.int32) - 1000
    npr = 5 * 4096 + 123
    pk = rng.integers(-3000, span + 2000, npr).astype(np.int32)
    for hint in (gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR),
                 gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, sort_mode=gx.SORTED_BUILD)):
        t = gx.inner_eq_join_rowids(to_dev(bk), to_dev(pk), hint)
        l, p = t.numpy_columns()
        o = np.lexsort((p, l))
        el, er = O.join_pairs(bk, pk)
        assert len(el) > npr // 3
        assert np.array_equal(l[o], el) and np.array_equal(p[o], er)


def test_join_many_to_many_and_wide_payloads():
    a = O.gen_keys(3000, np.int64, groups=500, seed=3)
    b = O.gen_keys(2000, np.int64, groups=700, seed=4)
    ap1 = O.gen_values(3000, np.int32, lo=0, hi=1 << 30, seed=5)
    ap2 = O.gen_values(3000, np.float64, seed=6)
    bp1 = O.gen_values(2000, np.int16, lo=-1000, hi=1000, seed=7)
    hint = gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR)
    t = gx.inner_eq_join([to_dev(a), to_dev(ap1), to_dev(ap2)], [to_dev(b), to_dev(bp1)], hint)
    key, c1, c2, c3 = t.numpy_columns()
    el, er = O.join_pairs(a, b)
    exp = np.stack([a[el], ap1[el].astype(np.int64), ap2[el].view(np.int64), bp1[er].astype(np.int64)])
    got = np.stack([key, c1.astype(np.int64), c2.view(np.int64), c3.astype(np.int64)])
    eo = np.lexsort(exp[::-1])
    go = np.lexsort(got[::-1])
    assert np.array_equal(got[:, go], exp[:, eo])


def test_join_edge_cases_and_validation():
    e = np.zeros(0, dtype=np.int32)
    x = np.array([1, 2, 3], dtype=np.int32)
    t = gx.inner_eq_join_rowids(to_dev(e), to_dev(x))
    assert t.num_rows == 0
    t = gx.inner_eq_join_rowids(to_dev(x), to_dev(np.array([4, 5], np.int32)))
    assert t.num_rows == 0
    with pytest.raises(gx.GxError):  # AUTO is rejected like check_join_solvable
        gx.inner_eq_join([to_dev(x), to_dev(x)], [to_dev(x), to_dev(x)], gx.make_join_hint(gx.JOIN_AUTO, gx.MAT_GFUR))
    with pytest.raises(gx.GxError):  # needs a payload column per side
        gx.inner_eq_join([to_dev(x)], [to_dev(x), to_dev(x)], gx.make_join_hint())
    with pytest.raises(gx.GxError):  # output larger than max_out
        gx.inner_eq_join([to_dev(x), to_dev(x)], [to_dev(x), to_dev(x)], gx.make_join_hint(max_out=2))


def test_join_full_size_property():
    # 2^24 unique build keys ⋈ 2^28 probe keys (10% absent): the match count
    # equals the present probe rows, and sampled pairs carry equal keys.
    import torch
    nb, npr = 1 << 24, 1 << 28
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    gx.generate_permutation(bk, 42)
    pk = torch.empty(npr, dtype=torch.int32, device="cuda")
    gx.generate_keys(pk, gx.gen_spec(seed=39, groups=nb, miss_frac=0.1))
    t = gx.inner_eq_join_rowids(bk, pk, gx.make_join_hint(unique_left=1))
    present = int((pk < nb).sum())
    assert t.num_rows == present
    l = t.to_torch(0)
    r = t.to_torch(1)
    sel = torch.randint(0, present, (1 << 16,), device="cuda")
    assert bool((bk[l[sel]] == pk[r[sel]]).all())
    assert bool((torch.bincount(r, minlength=npr) <= 1).all())


# ----------------------------------------------------------- dictionary ----
@pytest.mark.parametrize("kdt,et,ndv", [(np.int32, gx.INT32, 1), (np.int32, gx.INT32, 16), (np.int32, gx.INT32, 4096),
                                        (np.int64, gx.INT32, 16), (np.int64, gx.INT16, 256), (np.int64, gx.INT8, 100),
                                        (np.int32, gx.INT16, 256), (np.float64, gx.INT32, 16),
                                        (np.float32, gx.INT16, 256), (np.int64, gx.INT32, 1 << 16)])
def test_dictionary_encode(kdt, et, ndv):
    # dictionary_encode_test.cu:94-152 shapes at N = 4096 (plus 2^20 rows).
    for n in (4096, 1 << 20):
        base = O.gen_keys(n, np.int64, groups=ndv, scatter=1, seed=ndv)
        k = base.astype(kdt) if np.dtype(kdt).kind != "f" else (base % 1000003).astype(kdt) * kdt(0.25)
        codes, nd = gx.dictionary_encode(to_dev(k), et)
        c = codes.cpu().numpy().astype(np.int64)
        u = np.unique(k)
        assert nd == len(u)
        if et != gx.INT8 or nd <= 128:
            assert set(c.tolist()) == set(range(nd))
            assert len(set(zip(k.tolist(), c.tolist()))) == nd
        oc, nd2 = gx.dictionary_encode(to_dev(k), et, ordered=True)
        ec, _ = O.dict_encode(k, ordered=True)
        assert nd2 == nd
        assert np.array_equal(oc.cpu().numpy().astype(np.int64), ec.astype(np.dtype(gx._NP[et])).astype(np.int64))


def test_dictionary_encode_marker_key_and_ragged_rows():
    # INT64_MIN (the 8-byte table's empty marker, kept in a side slot) among
    # the keys, and a row count that leaves a partial round of rows per thread.
    n = (1 << 20) + 13
    k = O.gen_keys(n, np.int64, groups=3000, scatter=1, seed=77)
    k[::1001] = np.iinfo(np.int64).min
    codes, nd = gx.dictionary_encode(to_dev(k), gx.INT32)
    c = codes.cpu().numpy().astype(np.int64)
    assert nd == len(np.unique(k))
    assert set(c.tolist()) == set(range(nd))
    assert len(set(zip(k.tolist(), c.tolist()))) == nd
    oc, _ = gx.dictionary_encode(to_dev(k), gx.INT32, ordered=True)
    ec, _ = O.dict_encode(k, ordered=True)
    assert np.array_equal(oc.cpu().numpy().astype(np.int64), ec.astype(np.int64))
    d = np.unique(k)[::-1].copy()
    got = gx.dictionary_encode_with_dict(to_dev(k), to_dev(d)).cpu().numpy()
    assert np.array_equal(got, O.dict_with_dict(k, d))


def test_dictionary_encode_with_dict():
    d = O.gen_perm(4096, np.int32, seed=5, base=-2048)
    q = O.gen_keys(1 << 18, np.int32, groups=5000, seed=6) - 2048
    got = gx.dictionary_encode_with_dict(to_dev(q), to_dev(d)).cpu().numpy()
    assert np.array_equal(got, O.dict_with_dict(q, d))


# ------------------------------------------------------------ hll / gen ----
@pytest.mark.parametrize("kdt,G", [(np.int32, 1000), (np.int64, 1 << 18), (np.int32, 1 << 22)])
@pytest.mark.parametrize("extra", [0, 3])
def test_hll_matches_oracle_registers(kdt, G, extra):
    # extra = 3: a tail of keys past the last 16-byte vector.
    k = O.gen_keys((1 << 22) + extra, kdt, groups=G, scatter=1, seed=8)
    est = gx.compute_ndv_approx(to_dev(k))
    exp = O.hll_estimate(O.hll_registers(k))
    assert est == int(round(exp))
    assert abs(est - O.ndv_exact(k)) / O.ndv_exact(k) < 0.04


def test_hll_unaligned_view_and_narrow_keys():
    # A view starting one row into its buffer (not 16-byte aligned: the
    # strided kernel) and 16-bit keys (widened first): same registers as the
    # oracle.
    import torch
    k = O.gen_keys((1 << 20) + 1, np.int32, groups=5000, scatter=1, seed=9)
    d = to_dev(k)
    v = gx.ColumnView(d.data_ptr(), len(k) - 1, gx.INT32, 1)
    assert (d.data_ptr() + 4) % 16 != 0
    assert gx.compute_ndv_approx(v) == int(round(O.hll_estimate(O.hll_registers(k[1:]))))
    k16 = (k % 30000).astype(np.int16)
    assert gx.compute_ndv_approx(torch.from_numpy(k16).cuda()) == int(round(O.hll_estimate(O.hll_registers(k16))))


@pytest.mark.parametrize("dist,kdt", [(O.DIST_UNIFORM, np.int32), (O.DIST_CYCLIC, np.int64),
                                      (O.DIST_ZIPF, np.int32), (O.DIST_SEQUENCE, np.int64)])
def test_generators_match_cpu(dist, kdt):
    import torch
    n, G = 100003, 5000
    cdf = O.zipf_cdf(G, 1.2)
    dcdf = torch.from_numpy(cdf).cuda()
    k = torch.empty(n, dtype=torch.int32 if kdt == np.int32 else torch.int64, device="cuda")
    gx.generate_keys(k, gx.gen_spec(seed=3, stream_id=7, dist=dist, groups=G, scatter=1, zipf_s=1.2,
                                    zipf_cdf=dcdf.data_ptr(), miss_frac=0.05))
    exp = O.gen_keys(n, kdt, seed=3, stream_id=7, dist=dist, groups=G, scatter=1, zipf_s=1.2, miss_frac=0.05, cdf=cdf)
    assert np.array_equal(k.cpu().numpy(), exp)
    for vdt, lo, hi in ((np.int64, 0, 1 << 31), (np.float64, 0, 1), (np.int32, 100, 2557)):
        v = torch.empty(n, dtype=gx.torch_dtype(O.GX_OF_NP[np.dtype(vdt)]), device="cuda")
        gx.generate_values(v, gx.gen_spec(seed=4, stream_id=2, lo=lo, hi=hi))
        assert np.array_equal(v.cpu().numpy(), O.gen_values(n, vdt, seed=4, stream_id=2, lo=lo, hi=hi))
    p = torch.empty(4096, dtype=torch.int32, device="cuda")
    gx.generate_permutation(p, 11, -7)
    assert np.array_equal(p.cpu().numpy(), O.gen_perm(4096, np.int32, 11, -7))
    assert np.array_equal(gx.zipf_cdf(G, 1.2), cdf)


@pytest.mark.parametrize("algo", [gx.JOIN_HASH, gx.JOIN_PARTITION])
@pytest.mark.parametrize("mat", [gx.MAT_GFUR, gx.MAT_GFTR])
def test_join_hash_and_partition_hints_give_the_sort_result(algo, mat):
    # join_algo HASH / PARTITION (inner_join.cu:54-74) must return the same
    # pair multiset as SORT, including duplicate keys on both sides.
    lk = O.gen_keys(5000, np.int64, groups=700, seed=11)
    rk = O.gen_keys(20000, np.int64, groups=900, seed=12)
    lp = np.arange(5000, dtype=np.int64)
    rp = np.arange(20000, dtype=np.int64)
    t = gx.inner_eq_join([to_dev(lk), to_dev(lp)], [to_dev(rk), to_dev(rp)], gx.make_join_hint(algo, mat))
    cols = t.numpy_columns()
    got = np.lexsort((cols[2], cols[1]))
    el, er = O.join_pairs(lk, rk)
    assert np.array_equal(cols[1][got], el) and np.array_equal(cols[2][got], er)
