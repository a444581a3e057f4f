"""Host-side helpers of the selector and the batched engine, checked on the
CPU: instance drawing, training targets, chunk merging, regret, and the
string dictionary the batched-engine instances are built from."""
import json

import numpy as np

from eiger_b200 import batch, selector


def test_draw_instances_ranges_and_determinism():
    a = selector.draw_instances(200, seed=7)
    b = selector.draw_instances(200, seed=7)
    assert a == b
    assert selector.draw_instances(5, seed=8) != a[:5]
    for inst in a:
        assert 2 ** 16 <= inst["rows"] <= 2 ** 28
        assert 1 <= inst["ndv"] <= inst["rows"]
        assert 0.0 <= inst["zipf"] <= 2.0
        assert inst["key"] in ("int32", "int64")
    assert {inst["key"] for inst in a} == {"int32", "int64"}


def test_targets_mask_unmeasured_fanouts():
    times = np.array([[1.0, 2.0, 4.0], [8.0, 0.5, 2.0]])
    ftimes = np.array([[np.nan] * 4, [1.0, 2.0, np.nan, 4.0]])
    t, m = selector.targets_from(times, ftimes)
    assert t.shape == m.shape == (2, selector.O)
    assert np.allclose(t[:, :3], np.log2(times))
    assert np.all(m[:, :3] == 1)
    assert np.all(m[0, 3:] == 0)
    assert list(m[1, 3:]) == [1, 1, 0, 1]
    assert np.allclose(t[1, 3:][m[1, 3:] == 1], np.log2([1.0, 2.0, 4.0]))


def test_regret_is_relative_excess_over_the_best():
    times = np.array([[1.0, 2.0, 4.0], [3.0, 1.5, 6.0]])
    assert selector.regret(times, np.array([0, 1])) == 0.0
    assert np.isclose(selector.regret(times, np.array([1, 0])), (1.0 + 1.0) / 2)


def test_merge_orders_chunks_and_drops_duplicates(tmp_path):
    def chunk(idx, name):
        idx = np.array(idx)
        n = len(idx)
        insts = [{"rows": int(i)} for i in idx]
        path = tmp_path / name
        np.savez(path, index=idx, instances=json.dumps(insts), features=np.tile(idx[:, None], (1, 16)).astype(np.float32),
                 times=np.tile(idx[:, None], (1, 3)).astype(np.float64), fanout_times=np.full((n, 4), np.nan),
                 heuristic=idx.astype(np.int32))
        return str(path)

    out = selector.merge([chunk([4, 5, 6], "b.npz"), chunk([0, 1, 2, 3], "a.npz"), chunk([3, 4], "c.npz")])
    assert list(out["index"]) == [0, 1, 2, 3, 4, 5, 6]
    assert [i["rows"] for i in json.loads(out["instances"])] == [0, 1, 2, 3, 4, 5, 6]
    assert list(out["features"][:, 0]) == [0, 1, 2, 3, 4, 5, 6]
    assert list(out["heuristic"]) == [0, 1, 2, 3, 4, 5, 6]


def test_string_dictionary_is_distinct_ascii_with_arrow_offsets():
    chars, offs = batch.make_dictionary(2000, seed=3, min_len=8, max_len=32)
    assert offs.dtype == np.int64 and offs[0] == 0 and offs[-1] == len(chars)
    lens = np.diff(offs)
    assert lens.min() >= 8 and lens.max() <= 32
    assert chars.min() >= 33 and chars.max() <= 126
    words = {bytes(chars[offs[i]:offs[i + 1]]) for i in range(len(offs) - 1)}
    assert len(words) == 2000
    c2, o2 = batch.make_dictionary(2000, seed=3, min_len=8, max_len=32)
    assert np.array_equal(chars, c2) and np.array_equal(offs, o2)


def test_selector_support_holds_the_training_lists():
    # The plan features AUTO compares a request list with before it trusts
    # the network (host only): the two training lists, a near neighbour
    # inside the radius and a list with another accumulator mix outside it.
    import eiger_b200 as gx
    sup = selector.training_plan_support()
    assert np.allclose(sup, [[0.25, 0.125, 0.0, 0.0], [0.5, 0.75, 0.25, 0.5]])
    i32 = [gx.ColumnView(None, 0, gx.INT32, 0)]
    near = selector.plan_features(i32, [(0, gx.SUM), (0, gx.COUNT_ALL)])
    two = [gx.ColumnView(None, 0, gx.INT64, 0), gx.ColumnView(None, 0, gx.FLOAT64, 0)]
    far = selector.plan_features(two, [(1, gx.SUM), (0, gx.MAX), (0, gx.COUNT_ALL)])

    def dist(f):
        return float(np.abs(sup - f).max(axis=1).min())

    assert dist(near) <= selector.SUPPORT_RADIUS < dist(far)
    assert gx.lib.gx_selector_set_plan_support(None, -1, 0.1) != 0
    assert gx.lib.gx_selector_set_plan_support(sup.ctypes.data, len(sup), -1.0) != 0
