"""The multi-rank group-by and join of eiger_b200/distributed.py with the
library's own engine as the local step (not a stand-in), on one NCCL rank
on the GPU: the exchange degenerates to a local copy, so the result must be
the full group-by / join, checked against the oracle."""
import os
import socket

import numpy as np
import pytest

import eiger_b200 as gx
import oracle as O
from tests.helpers import to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_group():
    import torch
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    from datetime import timedelta
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60))
    yield
    dist.destroy_process_group()


def test_groupby_with_the_gpu_engine(nccl_group):
    from eiger_b200.distributed import distributed_groupby
    n = 1 << 20
    k = O.gen_keys(n, np.int32, groups=3000, scatter=1, seed=1)
    v = O.gen_values(n, np.int64, lo=-1000, hi=1000, seed=2)
    f = O.gen_values(n, np.float64, seed=3)
    reqs = [(0, gx.SUM), (1, gx.MAX), (0, gx.COUNT_ALL), (1, gx.AVG)]
    out = distributed_groupby(to_dev(k), [to_dev(v), to_dev(f)], reqs)
    got = [c.cpu().numpy() for c in out]
    o = np.argsort(got[0])
    exp = O.groupby(k, [v, f], [(0, O.SUM), (1, O.MAX), (0, O.COUNT_ALL), (1, O.AVG)])
    assert np.array_equal(got[0][o], exp[0])
    assert np.array_equal(got[1][o], exp[1]) and np.array_equal(got[2][o], exp[2])
    assert np.array_equal(got[3][o], exp[3])
    np.testing.assert_allclose(got[4][o], exp[4], rtol=1e-12, atol=0)


@pytest.mark.parametrize("strategy", ["broadcast", "shuffle"])
def test_join_with_the_gpu_engine(nccl_group, strategy):
    from eiger_b200.distributed import distributed_join
    bk = O.gen_perm(1 << 14, np.int32, seed=4)
    pk = O.gen_keys(1 << 18, np.int32, groups=1 << 14, seed=5, miss_frac=0.1)
    b, p = distributed_join(to_dev(bk), to_dev(pk), 0, 0, strategy=strategy)
    b, p = b.cpu().numpy(), p.cpu().numpy()
    o = np.lexsort((p, b))
    el, er = O.join_pairs(bk, pk)
    assert np.array_equal(b[o], el) and np.array_equal(p[o], er)
