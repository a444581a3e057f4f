"""Batched engine: one persistent CUDA-graph launch and the per-instance
plain engine both against the CPU restatement (oracle/batch.py), exact on
(string, SUM, COUNT) per group."""
import pytest

import oracle.batch as OB
from eiger_b200 import batch as B
import eiger_b200 as gx

pytestmark = pytest.mark.gpu


def expected(insts):
    return [OB.string_groupby(it.chars.cpu().numpy(), it.offsets.cpu().numpy(), it.date.cpu().numpy(),
                              it.amount.cpu().numpy(), it.lo, it.hi) for it in insts]


def test_batched_and_plain_match_oracle():
    insts, _ = B.make_instances(24, seed=3, min_log2=6, max_log2=14, dict_size=2000)
    exp = expected(insts)
    plan = B.Plan(insts, max_distinct=2000)
    t, lf = plan.tuning()
    assert t in (1024, 4096, 16384) and lf in (25, 50)
    for _ in range(2):  # graph capture, then replay
        plan.run()
        assert plan.results() == exp
    plan.run_per_instance()
    assert plan.results() == exp


def test_repeated_runs_of_one_plan():
    # Every run renumbers the strings (codes follow insertion order) and
    # rewrites the key store at the same addresses; a lookup must never
    # compare against bytes an earlier run left there (that inserts the
    # string again, and max_distinct = the dictionary size turns any second
    # insert into an overflow error).
    insts, _ = B.make_instances(64, seed=11, min_log2=12, max_log2=17, dict_size=3000)
    exp = expected(insts)
    plan = B.Plan(insts, max_distinct=3000)
    for _ in range(6):
        plan.run()
        assert plan.results() == exp


@pytest.mark.parametrize("keep", [0.0, 1.0])
def test_date_range_keeping_none_or_all(keep):
    # The batched launch applies the date range before encoding: a range
    # that keeps no row leaves every instance without groups, one that keeps
    # every row groups all of them; the per-instance engine (encode first)
    # agrees in both cases.
    insts, _ = B.make_instances(12, seed=23, min_log2=8, max_log2=14, dict_size=1500, keep=keep)
    exp = expected(insts)
    assert all(len(e) == 0 for e in exp) if keep == 0.0 else all(len(e) > 0 for e in exp)
    plan = B.Plan(insts, max_distinct=1500)
    plan.run()
    assert plan.results() == exp
    plan.run_per_instance()
    assert plan.results() == exp


def test_empty_and_tiny_instances():
    insts, _ = B.make_instances(5, seed=9, min_log2=0, max_log2=3, dict_size=50)
    plan = B.Plan(insts, max_distinct=50)
    plan.run()
    assert plan.results() == expected(insts)


def test_distinct_overflow_is_reported():
    insts, _ = B.make_instances(2, seed=4, min_log2=12, max_log2=12, dict_size=3000)
    plan = B.Plan(insts, max_distinct=100)
    with pytest.raises(gx.GxError):
        plan.run()


@pytest.mark.parametrize("size_hint", [0, 16])
def test_string_dictionary_encode_is_a_dense_bijection(size_hint):
    import numpy as np
    import torch
    dchars, doffs = B.make_dictionary(500, seed=21)
    d_dchars, d_doffs = torch.from_numpy(dchars).cuda(), torch.from_numpy(doffs).cuda()
    rows = 100_003
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    src = torch.randint(0, 400, (rows,), device="cuda", dtype=torch.int32, generator=g)  # 400 of 500 used
    offs = torch.zeros(rows + 1, dtype=torch.int64, device="cuda")
    torch.cumsum((d_doffs[1:] - d_doffs[:-1])[src.long()], 0, out=offs[1:])
    chars = torch.empty(int(offs[-1].item()), dtype=torch.uint8, device="cuda")
    gx.check(gx.lib.gx_generate_strings(d_dchars.data_ptr(), d_doffs.data_ptr(), 500, src.data_ptr(), rows,
                                        offs.data_ptr(), chars.data_ptr(), None))
    skip = 3  # a view that starts at row 3
    codes, ndv = gx.dictionary_encode_strings(chars, offs, row_offset=skip, size_hint=size_hint)
    s, c = src.cpu().numpy()[skip:], codes.cpu().numpy()
    assert len(c) == rows - skip and ndv == len(np.unique(s))
    assert c.min() == 0 and c.max() == ndv - 1 and len(np.unique(c)) == ndv
    # the same string <-> the same code, both ways
    pairs = np.unique(np.stack([s, c], 1), axis=0)
    assert len(pairs) == ndv


def test_string_dictionary_encode_empty():
    import torch
    offs = torch.zeros(1, dtype=torch.int64, device="cuda")
    chars = torch.zeros(1, dtype=torch.uint8, device="cuda")
    codes, ndv = gx.dictionary_encode_strings(chars, offs)
    assert codes.numel() == 0 and ndv == 0
