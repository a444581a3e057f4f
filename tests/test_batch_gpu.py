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
