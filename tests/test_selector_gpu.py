"""Learned selector: the FP16 MLP kernels against the NumPy restatement
(oracle/mlp.py), the sample sketch, training, and AUTO with learned weights."""
import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from oracle import mlp as M
from tests.helpers import assert_columns_match, sort_by_key, to_dev

pytestmark = pytest.mark.gpu


def rand_params(seed=0):
    rng = np.random.default_rng(seed)
    p = (rng.normal(0, 0.3, size=M.TOTAL)).astype(np.float16)
    return p


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_param_count_matches_layout():
    assert gx.lib.gx_selector_param_count() == M.TOTAL


def test_forward_matches_numpy():
    import torch
    p = rand_params(1)
    x = np.random.default_rng(2).normal(size=(37, M.F)).astype(np.float32)
    out = torch.empty((37, M.O), dtype=torch.float32, device="cuda")
    dp, dx = dev(p), dev(x)
    gx.check(gx.lib.gx_mlp_forward(dp.data_ptr(), dx.data_ptr(), 37, out.data_ptr(), None))
    exp = M.forward(p.astype(np.float64), x.astype(np.float64))
    np.testing.assert_allclose(out.cpu().numpy(), exp, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("rows", [1, 64, 1000])
def test_gradients_match_numpy(rows):
    import torch
    rng = np.random.default_rng(rows)
    p = rand_params(rows)
    x = rng.normal(size=(rows, M.F)).astype(np.float32)
    t = rng.normal(size=(rows, M.O)).astype(np.float32)
    mask = (rng.random((rows, M.O)) < 0.7).astype(np.float32)
    grads = torch.zeros(M.TOTAL, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    dp, dx, dt, dm = dev(p), dev(x), dev(t), dev(mask)
    gx.check(gx.lib.gx_mlp_forward_backward(dp.data_ptr(), dx.data_ptr(), dt.data_ptr(), dm.data_ptr(), rows,
                                            grads.data_ptr(), loss.data_ptr(), None))
    el, eg = M.forward_backward(p.astype(np.float64), x, t, mask)
    g = grads.cpu().numpy()
    assert abs(float(loss.item()) - el) <= 1e-4 * max(1.0, abs(el))
    np.testing.assert_allclose(g, eg, rtol=2e-3, atol=2e-4 * np.abs(eg).max())


def test_adam_step_matches_numpy():
    import torch
    rng = np.random.default_rng(5)
    master = rng.normal(size=M.TOTAL).astype(np.float32)
    g = rng.normal(size=M.TOTAL).astype(np.float32)
    m = np.zeros(M.TOTAL, np.float32)
    v = np.zeros(M.TOTAL, np.float32)
    dmaster, dg, dmm, dv = dev(master), dev(g), dev(m), dev(v)
    params = torch.empty(M.TOTAL, dtype=torch.float16, device="cuda")
    for step in (1, 2):
        gx.check(gx.lib.gx_mlp_adam_step(dmaster.data_ptr(), params.data_ptr(), dg.data_ptr(), dmm.data_ptr(),
                                         dv.data_ptr(), step, gx.C.c_float(1e-2), None))
        master, m, v = M.adam(master.astype(np.float64), g, m, v, step, 1e-2)
    np.testing.assert_allclose(dmaster.cpu().numpy(), master, rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(params.cpu().numpy(), dmaster.cpu().numpy().astype(np.float16))


def test_sample_sketch_features():
    from eiger_b200 import selector as S
    import torch
    same = torch.full((1 << 20,), 7, dtype=torch.int32, device="cuda")
    f = S.features(same)
    assert f[4] == pytest.approx(1.0 / 16384) and f[5] == 0 and f[6] == pytest.approx(1.0)
    uniq = torch.arange(1 << 20, dtype=torch.int64, device="cuda")
    f = S.features(uniq)
    assert f[1] == 1.0 and f[4] == pytest.approx(1.0) and f[5] == pytest.approx(1.0)
    # GEE (sqrt(N/n) * f1 + the rest) extrapolates past the sample's count.
    assert 2 ** (f[14] * 28) == pytest.approx(1 + 8 * 16384, rel=1e-4)


def test_training_reduces_loss():
    from eiger_b200 import selector as S
    rng = np.random.default_rng(0)
    x = rng.normal(size=(512, M.F)).astype(np.float32)
    w = rng.normal(size=(M.F, M.O)).astype(np.float32)
    t = np.tanh(x @ w).astype(np.float32)
    m = np.ones_like(t)
    params, hist = S.train(x, t, m, epochs=400, lr=3e-3)
    assert hist[-1][1] < 0.3 * hist[0][1]
    pred = S.predict(params, x)
    assert np.mean((pred - t) ** 2) < 0.3 * np.mean(t ** 2)


def test_auto_with_learned_selector_is_exact():
    from eiger_b200 import selector as S
    if not S.install():
        pytest.skip("no trained selector weights committed")
    n = 1 << 18
    for G in (100, 1 << 16):
        key = O.gen_keys(n, np.int32, groups=G, scatter=1, seed=G)
        val = O.gen_values(n, np.int64, lo=0, hi=1000, seed=3)
        hint = gx.make_hint(gx.AUTO_ALGO, selector=gx.SELECT_LEARNED)
        t = gx.groupby([to_dev(key)], [to_dev(val)], [(0, gx.SUM), (0, gx.COUNT_ALL)], hint)
        assert hint.groupby_algo in (gx.HASH, gx.SORT, gx.PARTITION)
        exp = O.groupby(key, [val], [(0, O.SUM), (0, O.COUNT_ALL)])
        assert_columns_match(sort_by_key(t.numpy_columns()), exp)


def test_auto_outside_the_trained_request_lists_uses_the_plain_rule():
    # A request list unlike the two the weights were trained on (here SUM f64
    # + MAX i64 + COUNT): AUTO does not extrapolate the network but takes the
    # plain NDV rule (<= 2^14 distinct 4-byte keys -> HASH, else PARTITION).
    from eiger_b200 import selector as S
    if not S.install():
        pytest.skip("no trained selector weights committed")
    n = 1 << 18
    iv = O.gen_values(n, np.int64, lo=0, hi=1 << 31, seed=71)
    fv = O.gen_values(n, np.float64, seed=72)
    reqs = [(1, gx.SUM), (0, gx.MAX), (0, gx.COUNT_ALL)]
    for G, want in ((1000, gx.HASH), (1 << 17, gx.PARTITION)):
        key = O.gen_keys(n, np.int32, groups=G, scatter=1, seed=73)
        hint = gx.make_hint(gx.AUTO_ALGO, selector=gx.SELECT_LEARNED)
        t = gx.groupby([to_dev(key)], [to_dev(iv), to_dev(fv)], reqs, hint)
        assert hint.groupby_algo == want
        exp = O.groupby(key, [iv, fv], [(1, O.SUM), (0, O.MAX), (0, O.COUNT_ALL)])
        assert_columns_match(sort_by_key(t.numpy_columns()), exp)
