"""Parity at the benchmarked sizes: the CUDA library against the CPU oracle
on the group-by sweep's 2^28-row configurations and the 2^24 x 2^28 join,
not only on the small cases of the other test files.

Inputs are generated on the device by the library's seeded generators and
copied to the host, so the oracle sees exactly the bytes the kernels read.
Group-by results are compared column by column after sorting by key:
keys, counts, integer SUM/MIN/MAX and float64 MIN/MAX bit-exact, float64
SUM within 1e-12 relative of the oracle's long double row-order sum.  Join
results (build_rowid, probe_rowid) of a unique build side are compared as
the full pair set: every probe row matches at most one build row, so the
pairs are exactly {(match[p], p) : match[p] >= 0} with match from the
oracle's probe.
"""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import assert_columns_match, sort_by_key

pytestmark = pytest.mark.gpu

ROWS = 1 << 28
REQS = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]
OREQS = [(0, O.SUM), (0, O.MIN), (0, O.MAX), (1, O.SUM), (1, O.MIN), (1, O.MAX), (0, O.COUNT_ALL)]


def make_groupby_inputs(kdt, groups, zipf_s, seed):
    """Device key column (scattered ranks, uniform or Zipf), int64 values in
    [0, 2^31) and float64 values in [0, 1), as the group-by sweep draws them."""
    import torch
    k = torch.empty(ROWS, dtype=torch.int32 if kdt == np.int32 else torch.int64, device="cuda")
    cdf = None
    if zipf_s > 0:
        cdf = torch.from_numpy(gx.zipf_cdf(groups, zipf_s)).cuda()
        spec = gx.gen_spec(seed=seed, dist=gx.DIST_ZIPF, groups=groups, zipf_s=zipf_s, scatter=1,
                           zipf_cdf=cdf.data_ptr())
    else:
        spec = gx.gen_spec(seed=seed, groups=groups, scatter=1)
    gx.generate_keys(k, spec)
    iv = torch.empty(ROWS, dtype=torch.int64, device="cuda")
    gx.generate_values(iv, gx.gen_spec(seed=seed, stream_id=1, lo=0, hi=1 << 31))
    fv = torch.empty(ROWS, dtype=torch.float64, device="cuda")
    gx.generate_values(fv, gx.gen_spec(seed=seed, stream_id=2))
    torch.cuda.synchronize()
    del cdf
    return k, iv, fv


class Case:
    """One 2^28-row configuration: device inputs plus the oracle's answer."""

    def __init__(self, kdt, groups, zipf_s, seed):
        self.k, self.iv, self.fv = make_groupby_inputs(kdt, groups, zipf_s, seed)
        self.groups = groups
        self.exp = O.groupby(self.k.cpu().numpy(), [self.iv.cpu().numpy(), self.fv.cpu().numpy()], OREQS)

    def check(self, algo, selector=gx.SELECT_HEURISTIC):
        hint = gx.make_hint(algo, self.groups, selector=selector)
        t = gx.groupby([self.k], [self.iv, self.fv], REQS, hint)
        got = sort_by_key(t.numpy_columns())
        del t
        assert_columns_match(got, self.exp)
        return hint

    def free(self):
        import torch
        del self.k, self.iv, self.fv, self.exp
        torch.cuda.empty_cache()


@pytest.fixture(scope="module")
def headline():
    c = Case(np.int32, 1 << 16, 0.0, 42)
    yield c
    c.free()


@pytest.mark.parametrize("algo", [gx.HASH, gx.SORT, gx.PARTITION, gx.PARTITION_GFUR, gx.SORT_GFUR])
def test_groupby_headline_2p28_rows_each_variant(headline, algo):
    # 2^28 rows, int32 keys uniform over 2^16 scattered values, int64 + float64
    # values, SUM / MIN / MAX on both and COUNT: the benchmark's step.
    hint = headline.check(algo)
    assert hint.groupby_algo == algo
    assert len(headline.exp[0]) == 1 << 16


def test_groupby_headline_2p28_rows_auto_learned(headline):
    from eiger_b200 import selector
    assert selector.install()
    hint = headline.check(gx.AUTO_ALGO, selector=gx.SELECT_LEARNED)
    assert hint.groupby_algo in (gx.HASH, gx.SORT, gx.PARTITION)


@pytest.mark.parametrize("kdt,groups,zipf_s", [(np.int64, 1 << 20, 1.5), (np.int64, 1 << 24, 1.5),
                                               (np.int32, 1 << 26, 0.0)])
def test_groupby_2p28_rows_hard_corners(kdt, groups, zipf_s):
    # Zipf 1.5 puts ~38% of all rows on one key (its float64 SUM adds about
    # 10^8 values); 2^26 uniform groups leave ~4 rows per group.
    c = Case(kdt, groups, zipf_s, 7)
    try:
        if zipf_s > 0:
            assert c.exp[7].max() > ROWS // 4  # the heavy hitter is there
        for algo in (gx.HASH, gx.SORT, gx.PARTITION):
            c.check(algo)
    finally:
        c.free()


# ---------------------------------------------------------------- join ----
def check_unique_build_join(bk, pk, hint):
    """Full pair-set check of a join whose build side (left) has unique keys."""
    import torch
    t = gx.inner_eq_join_rowids(bk, pk, hint)
    l = t.to_torch(0)
    r = t.to_torch(1)
    match = torch.from_numpy(O.join_probe_unique(bk.cpu().numpy(), pk.cpu().numpy())).cuda()
    hit = match >= 0
    assert t.num_rows == int(hit.sum())
    # Each probe row at most once, and its build row is the oracle's match.
    got = torch.full_like(match, -1)
    got[r] = l
    assert bool((torch.bincount(r, minlength=pk.numel()) <= 1).all())
    assert torch.equal(got, match)
    assert bool((bk[l] == pk[r]).all())
    return t.num_rows


def test_join_2p28_probe_zipf_1():
    # 2^24 unique build keys (a permutation of 0..2^24-1); 2^28 probe keys
    # drawn Zipf s = 1.0 over the build keys (rank r -> the r-th build key).
    import torch
    nb, npr = 1 << 24, 1 << 28
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    gx.generate_permutation(bk, 42)
    cdf = torch.from_numpy(gx.zipf_cdf(nb, 1.0)).cuda()
    zr = torch.empty(npr, dtype=torch.int32, device="cuda")
    gx.generate_keys(zr, gx.gen_spec(seed=41, dist=gx.DIST_ZIPF, groups=nb, zipf_s=1.0, zipf_cdf=cdf.data_ptr()))
    pk = bk[zr.long()]
    del zr, cdf
    m = check_unique_build_join(bk, pk, gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, unique_left=1))
    assert m == npr


@pytest.mark.parametrize("algo", [gx.JOIN_HASH, gx.JOIN_PARTITION])
def test_join_2p28_probe_hash_plans(algo):
    # The benchmark's join (2^24 unique build keys, 2^28 probe keys, 10%
    # absent) through the hash multiset and the partitioned hash join.
    import torch
    nb, npr = 1 << 24, 1 << 28
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    gx.generate_permutation(bk, 42)
    pk = torch.empty(npr, dtype=torch.int32, device="cuda")
    gx.generate_keys(pk, gx.gen_spec(seed=39, groups=nb, miss_frac=0.1))
    m = check_unique_build_join(bk, pk, gx.make_join_hint(algo, gx.MAT_GFUR, unique_left=1))
    assert abs(m - 0.9 * npr) < 0.01 * npr


@pytest.mark.parametrize("mode", [gx.SORTED_BUILD, gx.SORT_MERGE])
def test_join_2p28_probe_sorted_build_matcher(mode):
    # Unique build keys 8 * perm(2^24): they span 2^27 values, too sparse for
    # the dense placement path, so the sorted-build matcher (or the full
    # sort-merge) runs.  Probe: 8 * rank with 10% of ranks past the build
    # range (absent).
    import torch
    nb, npr = 1 << 24, 1 << 28
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    gx.generate_permutation(bk, 43)
    bk *= 8
    pk = torch.empty(npr, dtype=torch.int32, device="cuda")
    gx.generate_keys(pk, gx.gen_spec(seed=44, groups=nb, miss_frac=0.1))
    pk *= 8
    m = check_unique_build_join(bk, pk, gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, unique_left=1, sort_mode=mode))
    assert abs(m - 0.9 * npr) < 0.01 * npr
