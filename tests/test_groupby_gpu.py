"""Group-by parity: the CUDA library (through its C ABI) against the CPU
oracle, for every variant (HASH, SORT, SORT_OPT, SORT_GFUR, PARTITION,
PARTITION_GFUR, AUTO), key/value dtypes, aggregations and key
distributions, plus the edge cases the reference's tests cover.  Integer
results are compared bit-exact after sorting by key; float64 SUM / AVG
within 1e-12 relative."""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import assert_columns_match, sort_by_key, to_dev

pytestmark = pytest.mark.gpu

VARIANTS = [gx.HASH, gx.SORT, gx.SORT_OPT, gx.SORT_GFUR, gx.PARTITION, gx.PARTITION_GFUR]
OKIND = {gx.SUM: O.SUM, gx.MIN: O.MIN, gx.MAX: O.MAX, gx.AVG: O.AVG, gx.ANY: O.ANY, gx.COUNT_ALL: O.COUNT_ALL}


def run_both(key, vals, reqs, algo, bound=None, agg_count=False, **hint_kw):
    hint = gx.make_hint(algo, bound, agg_count=int(agg_count), **hint_kw)
    t = gx.groupby([to_dev(key)], [to_dev(v) for v in vals], reqs, hint)
    got = sort_by_key(t.numpy_columns())
    exp = O.groupby(key, vals, [(c, OKIND[k]) for c, k in reqs], agg_count=agg_count)
    return got, exp, hint


@pytest.mark.parametrize("algo", VARIANTS)
def test_c1_hash_groupby_config(algo):
    # 2^20 rows, int32 keys uniform over 1024 values, int64 values in [0, 1e6), SUM + COUNT.
    n = 1 << 20
    key = O.gen_keys(n, np.int32, groups=1024, seed=42, stream_id=0)
    val = O.gen_values(n, np.int64, lo=0, hi=1_000_000, seed=42, stream_id=1)
    got, exp, _ = run_both(key, [val], [(0, gx.SUM), (0, gx.COUNT_ALL)], algo, bound=1024)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("algo", VARIANTS)
@pytest.mark.parametrize("kdt", [np.int32, np.int64])
@pytest.mark.parametrize("G,dist,s", [(16, O.DIST_UNIFORM, 0.0), (5000, O.DIST_UNIFORM, 0.0),
                                      (1 << 17, O.DIST_UNIFORM, 0.0), (4096, O.DIST_ZIPF, 1.0),
                                      (1 << 16, O.DIST_ZIPF, 1.5)])
def test_sweep_all_aggregates(algo, kdt, G, dist, s):
    n = 1 << 18
    key = O.gen_keys(n, kdt, dist=dist, groups=G, zipf_s=s, scatter=1, seed=5)
    iv = O.gen_values(n, np.int64, lo=0, hi=1 << 31, seed=6)
    fv = O.gen_values(n, np.float64, seed=7)
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]
    got, exp, hint = run_both(key, [iv, fv], reqs, algo, bound=G)
    assert_columns_match(got, exp)
    assert hint.groupby_algo == (gx.SORT_OPT if algo == gx.SORT_OPT else algo)


@pytest.mark.parametrize("algo", VARIANTS)
def test_unknown_bound_high_cardinality(algo):
    # No groups_upper_bound: the engine sizes its tables itself.
    n = 1 << 18
    key = O.gen_keys(n, np.int32, groups=1 << 17, scatter=1, seed=8)
    val = O.gen_values(n, np.int64, lo=-100, hi=100, seed=9)
    got, exp, _ = run_both(key, [val], [(0, gx.SUM), (0, gx.MAX)], algo)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("algo", VARIANTS)
@pytest.mark.parametrize("vdt", [np.int8, np.int16, np.int32, np.uint32, np.float32, np.int64, np.float64])
def test_value_types(algo, vdt):
    n = 20000
    key = O.gen_keys(n, np.int64, groups=300, scatter=1, seed=10)
    if np.dtype(vdt).kind == "f":
        val = (O.gen_values(n, np.float64, seed=11) * 200 - 100).astype(vdt)
    else:
        info = np.iinfo(vdt)
        val = O.gen_values(n, np.int64, lo=max(info.min, -(1 << 30)), hi=min(info.max, 1 << 30), seed=11).astype(vdt)
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (0, gx.AVG)]
    got, exp, _ = run_both(key, [val], reqs, algo, bound=300)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("algo", VARIANTS)
@pytest.mark.parametrize("kdt", [np.int8, np.int16, np.uint32, np.uint64, np.float32, np.float64])
def test_key_types(algo, kdt):
    n = 30000
    if np.dtype(kdt).kind == "f":
        key = (O.gen_keys(n, np.int64, groups=200, seed=12).astype(np.float64) - 100).astype(kdt) * kdt(0.5)
    else:
        key = O.gen_keys(n, np.int64, groups=120, seed=12).astype(kdt)
    val = O.gen_values(n, np.int64, lo=0, hi=1000, seed=13)
    got, exp, _ = run_both(key, [val], [(0, gx.SUM), (0, gx.COUNT_ALL)], algo)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("algo", VARIANTS)
def test_edge_cases(algo):
    cases = {
        "one_row": np.array([7], dtype=np.int64),
        "single_group": np.full(10000, -3, dtype=np.int64),
        "all_unique": np.arange(50000, dtype=np.int64)[::-1].copy(),
        "negative": np.array([-1, -2, -1, 5, -2, 5, 0], dtype=np.int64),
        "sentinel_keys": np.array([np.iinfo(np.int64).min, 0, np.iinfo(np.int64).min, -1, np.iinfo(np.int64).max],
                                  dtype=np.int64),
        "int32_extremes": np.array([np.iinfo(np.int32).min, -1, np.iinfo(np.int32).max, -1], dtype=np.int32),
    }
    for name, key in cases.items():
        val = np.arange(len(key), dtype=np.int64) * 3 - 7
        got, exp, _ = run_both(key, [val], [(0, gx.SUM), (0, gx.MIN), (0, gx.COUNT_ALL)], algo)
        assert_columns_match(got, exp)


@pytest.mark.parametrize("algo", VARIANTS)
def test_empty_input(algo):
    key = np.zeros(0, dtype=np.int32)
    val = np.zeros(0, dtype=np.int64)
    import torch
    hint = gx.make_hint(algo)
    t = gx.groupby([torch.zeros(0, dtype=torch.int32, device="cuda")],
                   [torch.zeros(0, dtype=torch.int64, device="cuda")], [(0, gx.SUM)], hint)
    assert t.num_rows == 0 and t.num_columns == 2
    assert t.type(1) == gx.INT64


def test_float_zero_keys_merge():
    key = np.array([0.0, -0.0, 1.5, -0.0, 1.5], dtype=np.float64)
    val = np.arange(5, dtype=np.int64)
    for algo in VARIANTS:
        got, exp, _ = run_both(key, [val], [(0, gx.SUM)], algo)
        assert len(got[0]) == 2
        assert np.array_equal(got[1], exp[1])


def test_agg_count_hint_and_avg_layout():
    # Output layout follows groupby.cu:346-392: [key, requests..., count].
    key = np.array([1, 1, 2, 2, 2], dtype=np.int32)
    val = np.array([10, 20, 30, 40, 50], dtype=np.int32)
    for algo in VARIANTS:
        got, exp, _ = run_both(key, [val], [(0, gx.AVG), (0, gx.SUM)], algo, agg_count=True)
        assert [g.dtype for g in got] == [np.int32, np.float64, np.int64, np.int64]
        assert_columns_match(got, exp)


def test_auto_heuristic_choice():
    # groupby.cu:99-118: NDV <= 2^14 (4-byte keys) -> HASH, else PARTITION.
    n = 1 << 18
    low = O.gen_keys(n, np.int32, groups=1000, seed=1)
    high = O.gen_keys(n, np.int32, groups=1 << 17, scatter=1, seed=1)
    val = np.ones(n, dtype=np.int64)
    for key, want in ((low, gx.HASH), (high, gx.PARTITION)):
        hint = gx.make_hint(gx.AUTO_ALGO)
        gx.groupby([to_dev(key)], [to_dev(val)], [(0, gx.SUM)], hint)
        assert hint.groupby_algo == want


def test_any_returns_a_group_member():
    n = 10000
    key = O.gen_keys(n, np.int32, groups=50, seed=3)
    val = O.gen_values(n, np.int64, lo=0, hi=1 << 40, seed=4)
    for algo in VARIANTS:
        t = gx.groupby([to_dev(key)], [to_dev(val)], [(0, gx.ANY)], gx.make_hint(algo, 50))
        k, a = t.numpy_columns()
        for kk, aa in zip(k, a):
            assert aa in set(val[key == kk].tolist())


def test_partition_radix_bits_and_overflow_spill():
    # A tiny fan-out forces partitions past their shared-table capacity; the
    # spill path must still produce exact results (the reference throws).
    n = 1 << 18
    key = O.gen_keys(n, np.int64, groups=1 << 16, scatter=1, seed=21)
    val = O.gen_values(n, np.int64, lo=0, hi=100, seed=22)
    for bits in (1, 4, 9, 16):
        got, exp, hint = run_both(key, [val], [(0, gx.SUM), (0, gx.COUNT_ALL)], gx.PARTITION, radix_bits=bits)
        assert hint.radix_bits == bits
        assert_columns_match(got, exp)


@pytest.mark.parametrize("kdt", [np.int32, np.int64])
@pytest.mark.parametrize("slot_table", [False, True])
def test_partition_units_spill_when_tables_run_out(monkeypatch, slot_table, kdt):
    # A group bound of 2^10 with 16 partitions sizes the unit tables for ~64
    # groups per partition; each partition holds ~2048.  The dense-id kernel
    # runs out of ids (the slot-indexed one closes its table): the remaining
    # keys go to the global table and the units merge there.
    if slot_table:
        monkeypatch.setenv("GX_UNITS_SLOT_TABLE", "1")
    n = 1 << 18
    key = O.gen_keys(n, kdt, groups=1 << 15, scatter=1, seed=23)
    iv = O.gen_values(n, np.int64, lo=-(1 << 35), hi=1 << 35, seed=24)
    fv = O.gen_values(n, np.float64, seed=25)
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]
    got, exp, hint = run_both(key, [iv, fv], reqs, gx.PARTITION, bound=1 << 10, radix_bits=4)
    assert hint.radix_bits == 4
    assert len(got[0]) == len(exp[0]) > 30000
    assert_columns_match(got, exp)


def test_closed_form_uniform_2_28_property():
    # Full-size property check (groupby_test.hpp:64-74): 2^26 rows of
    # shuffled i % G keys with all-ones values; every group sums to N/G.
    import torch
    n, G = 1 << 26, 1 << 20
    k = torch.empty(n, dtype=torch.int32, device="cuda")
    gx.generate_keys(k, gx.gen_spec(seed=1, dist=gx.DIST_CYCLIC, groups=G))
    ones = torch.ones(n, dtype=torch.int32, device="cuda")
    for algo in (gx.HASH, gx.PARTITION, gx.SORT):
        t = gx.groupby([k], [ones, ones], [(0, gx.SUM), (1, gx.SUM)], gx.make_hint(algo, G))
        keys, s0, s1 = t.numpy_columns()
        assert len(keys) == G
        assert np.all(s0 == n // G) and np.all(s1 == n // G)
        assert int(keys.astype(np.int64).sum()) == G * (G - 1) // 2


@pytest.mark.parametrize("kdt,bits", [(np.int32, 8), (np.int64, 12)])
@pytest.mark.parametrize("algo", [gx.PARTITION, gx.PARTITION_GFUR])
def test_partition_bulk_scatter_matches_register_scatter(monkeypatch, kdt, bits, algo):
    # Several tiles per SM plus a partial last tile, through the bulk-copy
    # scatter and through the register scatter (GX_PART_NO_BULK): both must
    # match the oracle (float sums within tolerance: shared-memory atomics
    # add in no fixed order).
    import torch
    n = 148 * 3 * 4096 + 1234
    key = O.gen_keys(n, kdt, groups=1 << 16, scatter=1, seed=31)
    iv = O.gen_values(n, np.int64, lo=-(1 << 40), hi=1 << 40, seed=32)
    fv = O.gen_values(n, np.float64, seed=33)
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]

    def run(kt, it, ft):
        hint = gx.make_hint(algo, 1 << 16, radix_bits=bits)
        return sort_by_key(gx.groupby([kt], [it, ft], reqs, hint).numpy_columns())

    kt, it, ft = to_dev(key), to_dev(iv), to_dev(fv)
    bulk = run(kt, it, ft)
    monkeypatch.setenv("GX_PART_NO_BULK", "1")
    reg = run(kt, it, ft)
    monkeypatch.delenv("GX_PART_NO_BULK")
    exp = O.groupby(key, [iv, fv], [(c, OKIND[k]) for c, k in reqs])
    assert_columns_match(bulk, exp)
    assert_columns_match(reg, exp)
    # A value column that starts 8 bytes into its buffer cannot be copied in
    # 16-byte units: the register scatter takes it, same results.
    shifted = torch.from_numpy(np.concatenate([np.zeros(1, np.int64), iv])).cuda()[1:]
    assert shifted.data_ptr() % 16 == 8
    assert_columns_match(run(kt, shifted, ft), exp)


@pytest.mark.parametrize("order", ["decreasing", "increasing", "mixed"])
def test_partition_min_max_monotone_values(order):
    # The unit aggregation reads a group's MIN/MAX and takes the atomic only
    # when the row moves the extreme.  Monotone values make every late row a
    # new extreme (or none of them); floats carry NaN, -0.0 / +0.0 and
    # infinities.
    n, G = 1 << 20, 4096
    key = O.gen_keys(n, np.int32, groups=G, scatter=1, seed=41)
    idx = np.arange(n, dtype=np.int64)
    if order == "decreasing":
        iv = -idx * 3 + 7
    elif order == "increasing":
        iv = idx * 5 - (1 << 40)
    else:
        iv = np.where(idx % 2 == 0, idx, -idx) * 11
    fv = O.gen_values(n, np.float64, seed=42) + 0.5  # positive: float SUMs without cancellation
    fv = fv * (1.0 + idx / n) if order != "decreasing" else fv * (2.0 - idx / n)
    special = np.array([np.nan, -0.0, 0.0, np.inf, -np.inf], dtype=np.float64)
    pick = (idx % 997) == 0
    fv[pick] = special[(idx[pick] // 997) % len(special)]
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]
    hint = gx.make_hint(gx.PARTITION, G)
    got = sort_by_key(gx.groupby([to_dev(key)], [to_dev(iv), to_dev(fv)], reqs, hint).numpy_columns())
    exp = O.groupby(key, [iv, fv], [(c, OKIND[k]) for c, k in reqs])
    # MIN / MAX exact (no rounding is involved).  Float extremes compare by
    # value: a group holding both zeros may keep either sign (the device
    # orders -0.0 below +0.0, the oracle keeps the first seen).
    for c in (2, 3):
        assert np.array_equal(got[c], exp[c]), c
    for c in (5, 6):
        assert np.array_equal(got[c], exp[c], equal_nan=True), c
    assert_columns_match(got, exp)


@pytest.mark.parametrize("kdt", [np.int32, np.int64])
@pytest.mark.parametrize("slot_table", [False, True])
@pytest.mark.parametrize("pattern", ["late_extremes", "decreasing"])
def test_partition_min_max_large_units(monkeypatch, pattern, slot_table, kdt):
    # Units of ~56K rows (2^26 rows, 2^12 groups), through the dense-id unit
    # kernel and the slot-indexed one (GX_UNITS_SLOT_TABLE).
    # "late_extremes" plants every group's true MIN and MAX (and float NaN,
    # infinities, signed zeros, int64 limits) in the last eighth of the rows,
    # long after each group's first rows; "decreasing" makes every row a new
    # MIN.
    if slot_table:
        monkeypatch.setenv("GX_UNITS_SLOT_TABLE", "1")
    n, G = 1 << 26, 1 << 12
    key = O.gen_keys(n, kdt, groups=G, scatter=1, seed=43)
    idx = np.arange(n, dtype=np.int64)
    if pattern == "decreasing":
        iv = (n - idx) * 7 - (1 << 33)
        fv = 1.0e6 - idx * 0.25
    else:
        rng = np.random.default_rng(44)
        iv = rng.integers(-(1 << 40), 1 << 40, n, dtype=np.int64)
        fv = rng.random(n) + 0.5  # positive: float SUMs without cancellation
        late = idx >= n - n // 8
        pick = late & (rng.random(n) < 0.002)
        m = int(pick.sum())
        iv[pick] = np.where(rng.random(m) < 0.5, -(1 << 50), 1 << 50) + rng.integers(-1000, 1000, m)
        fv[pick] = np.where(rng.random(m) < 0.5, -50.0, 50.0) * (1.0 + rng.random(m))
        ends = np.nonzero(late & ~pick)[0]
        e = rng.choice(ends, 64, replace=False)
        iv[e[:8]] = np.iinfo(np.int64).min
        iv[e[8:16]] = np.iinfo(np.int64).max
        fv[e[16:24]] = -np.inf
        fv[e[24:32]] = np.inf
        fv[e[32:40]] = np.nan
        fv[e[40:52]] = -0.0
        fv[e[52:64]] = 0.0
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]
    hint = gx.make_hint(gx.PARTITION, G)
    got = sort_by_key(gx.groupby([to_dev(key)], [to_dev(iv), to_dev(fv)], reqs, hint).numpy_columns())
    assert hint.groupby_algo == gx.PARTITION
    exp = O.groupby(key, [iv, fv], [(c, OKIND[k]) for c, k in reqs])
    for c in (0, 2, 3, 7):
        assert np.array_equal(got[c], exp[c]), c
    for c in (5, 6):
        assert np.array_equal(got[c], exp[c], equal_nan=True), c
    if pattern == "late_extremes":
        # the planted values are the extremes of the groups that got one
        assert (got[2] <= -(1 << 50) + 1000).sum() > G // 4
        assert (got[5] <= -50.0).sum() > G // 4
    # Integer SUM wraps identically; float SUM within tolerance (or NaN / inf
    # where the group holds one).
    assert_columns_match(got, exp)


@pytest.mark.parametrize("env,algo,G", [
    ("GX_HASH_GENERIC", gx.HASH, 4096),      # run-time aggregation list instead of a compiled plan
    ("GX_HASH_GENERIC", gx.PARTITION, 1 << 16),
    ("GX_HASH_GENERIC+GX_UNITS_SLOT_TABLE", gx.PARTITION, 1 << 16),  # run-time list, slot-indexed unit tables
    ("GX_HASH_GENERIC+GX_HASH_NO_UNITS", gx.HASH, 1024),  # run-time list, HASH's shared-table kernel
    ("GX_PART_OLD_AGG", gx.PARTITION, 1 << 16),  # per-partition CTA aggregation kernel
    ("GX_UNITS_SLOT_TABLE", gx.PARTITION, 1 << 16),  # slot-indexed unit tables instead of dense group ids
    ("GX_HASH_NO_UNITS", gx.HASH, 1024),  # HASH's shared-table kernel instead of dense-id units on row ranges
    ("GX_HASH_NO_UNITS", gx.HASH, 2048),
])
def test_forced_alternative_kernels(monkeypatch, env, algo, G):
    # The switches route a plan through its alternative kernel; results must
    # not change.
    n = 1 << 19
    key = O.gen_keys(n, np.int32, groups=G, scatter=1, seed=51)
    iv = O.gen_values(n, np.int64, lo=-(1 << 35), hi=1 << 35, seed=52)
    fv = O.gen_values(n, np.float64, seed=53)
    reqs = [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]
    for e in env.split("+"):
        monkeypatch.setenv(e, "1")
    got, exp, _ = run_both(key, [iv, fv], reqs, algo, bound=G)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("ncols", [3, 5])
@pytest.mark.parametrize("algo,G", [(gx.HASH, 1024), (gx.PARTITION, 1 << 16), (gx.AUTO_ALGO, 1 << 16)])
def test_many_value_columns(algo, G, ncols):
    # Run-time aggregation lists over three or five value columns of mixed
    # widths: the dense-id unit kernel takes up to four columns, the
    # slot-indexed one (or HASH's shared-table kernel) more; PARTITION moves
    # four columns (24 B per row) through the bulk-copy scatter and six
    # through the register-staged one.
    n = (1 << 19) + 77
    key = O.gen_keys(n, np.int32, groups=G, scatter=1, seed=61)
    cols = [O.gen_values(n, np.int64, lo=-(1 << 40), hi=1 << 40, seed=62),
            O.gen_values(n, np.float64, seed=63),
            O.gen_values(n, np.int32, lo=-(1 << 20), hi=1 << 20, seed=64),
            O.gen_values(n, np.float32, seed=65),
            O.gen_values(n, np.int16, lo=-1000, hi=1000, seed=66)][:ncols]
    reqs = [(0, gx.SUM), (1, gx.SUM), (2, gx.MIN), (2, gx.MAX), (0, gx.COUNT_ALL)]
    if ncols == 5:
        reqs += [(3, gx.MAX), (4, gx.SUM), (4, gx.MIN)]
    got, exp, _ = run_both(key, cols, reqs, algo, bound=G)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("bits", [8, 12])
def test_partition_four_moved_columns(bits):
    # Key + three 4-byte value columns (16 B per row): the bulk-copy scatter
    # with four moved columns, over 12 radix bits in two passes (the second
    # with the stable ranking).
    n = (1 << 19) + 77
    key = O.gen_keys(n, np.int32, groups=1 << 16, scatter=1, seed=81)
    cols = [O.gen_values(n, np.int32, lo=-(1 << 30), hi=1 << 30, seed=82 + i) for i in range(3)]
    reqs = [(0, gx.SUM), (1, gx.MIN), (2, gx.MAX), (0, gx.COUNT_ALL)]
    got, exp, _ = run_both(key, cols, reqs, gx.PARTITION, bound=1 << 16, radix_bits=bits)
    assert_columns_match(got, exp)


@pytest.mark.parametrize("smem", ["0", "1"])
def test_hash_table_mode_forced(monkeypatch, smem):
    # GX_HASH_SMEM forces the HASH plan's shared-table mode on or off (global
    # L2-resident record table only).
    n = 1 << 19
    key = O.gen_keys(n, np.int64, groups=3000, scatter=1, seed=61)
    val = O.gen_values(n, np.int64, lo=0, hi=1 << 20, seed=62)
    monkeypatch.setenv("GX_HASH_SMEM", smem)
    got, exp, _ = run_both(key, [val], [(0, gx.SUM), (0, gx.MAX), (0, gx.COUNT_ALL)], gx.HASH, bound=3000)
    assert_columns_match(got, exp)


def test_partition_groups_per_partition_override(monkeypatch):
    # GX_PART_GROUPS sets the target groups per partition (here 16: more radix
    # bits, two digit passes at this group count).
    n = 1 << 19
    key = O.gen_keys(n, np.int32, groups=1 << 16, scatter=1, seed=71)
    val = O.gen_values(n, np.int64, lo=0, hi=1000, seed=72)
    monkeypatch.setenv("GX_PART_GROUPS", "16")
    got, exp, hint = run_both(key, [val], [(0, gx.SUM), (0, gx.COUNT_ALL)], gx.PARTITION, bound=1 << 16)
    assert hint.radix_bits == 12
    assert_columns_match(got, exp)
