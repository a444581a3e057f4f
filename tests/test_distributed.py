"""The multi-rank group-by exchange (eiger_b200/distributed.py) on two gloo
ranks on the CPU: each rank holds a row shard, the local aggregation is the
oracle (standing in for the GPU engine), and the merged result each rank owns
must equal the oracle's group-by of all rows restricted to that rank's keys."""
import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

N, G, WORLD = 20_000, 700, 2
SUM, MAX, MIN, AVG, ANY, COUNT_ALL = range(6)
REQS = [(0, SUM), (0, COUNT_ALL), (1, MIN), (2, MAX), (1, AVG), (2, SUM)]


def full_data():
    import oracle as O
    k = O.gen_keys(N, np.int32, seed=5, groups=G, scatter=1)
    v0 = O.gen_values(N, np.int64, seed=5, stream_id=1, lo=-1000, hi=1000)
    v1 = O.gen_values(N, np.int32, seed=5, stream_id=2, lo=-50, hi=50)
    v2 = O.gen_values(N, np.float64, seed=5, stream_id=3)
    return k, [v0, v1, v2]


def oracle_local(keys, vals, requests):
    import torch
    import oracle as O
    cols = O.groupby(keys.numpy(), [v.numpy() for v in vals], requests)
    return [torch.from_numpy(np.ascontiguousarray(c)) for c in cols]


def worker(rank, rdv, failures):
    import torch
    import torch.distributed as dist
    import oracle as O
    from eiger_b200.distributed import distributed_groupby, destination
    try:
        dist.init_process_group("gloo", init_method=f"file://{rdv}", rank=rank, world_size=WORLD)
        k, vals = full_data()
        lo, hi = rank * N // WORLD, (rank + 1) * N // WORLD
        mine = [torch.from_numpy(a[lo:hi].copy()) for a in [k] + vals]
        out = distributed_groupby(mine[0], mine[1:], REQS, local_groupby=oracle_local)
        exp = O.groupby(k, vals, REQS)
        own = destination(torch.from_numpy(exp[0]), WORLD).numpy() == rank
        order = np.argsort(out[0].numpy(), kind="stable")
        got = [c.numpy()[order] for c in out]
        assert np.array_equal(got[0], exp[0][own])
        for j, (col, kind) in enumerate(REQS):
            e = exp[1 + j][own]
            if got[1 + j].dtype.kind == "f":
                np.testing.assert_allclose(got[1 + j], e, rtol=1e-12, atol=0)
            else:
                assert got[1 + j].dtype == e.dtype and np.array_equal(got[1 + j], e), (j, kind)
        # every rank owns something and the owners partition the keys
        counts = torch.tensor([len(got[0])], dtype=torch.int64)
        dist.all_reduce(counts)
        assert int(counts.item()) == len(exp[0])
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        failures.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


def test_two_rank_groupby_matches_single_oracle():
    ctx = mp.get_context("spawn")
    failures = ctx.SimpleQueue()
    with tempfile.TemporaryDirectory() as d:
        rdv = os.path.join(d, "rdv")
        procs = [ctx.Process(target=worker, args=(r, rdv, failures)) for r in range(WORLD)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        for p in procs:
            if p.is_alive():
                p.kill()
    msgs = []
    while not failures.empty():
        msgs.append(failures.get())
    assert not msgs, msgs
    assert all(p.exitcode == 0 for p in procs)


def test_split_requests_rewrites_avg_and_count():
    from eiger_b200.distributed import split_requests
    local, merge, finals = split_requests([(0, AVG), (1, COUNT_ALL), (2, MAX)])
    assert local == [(0, SUM), (0, COUNT_ALL), (1, COUNT_ALL), (2, MAX)]
    assert merge == [(0, SUM), (1, SUM), (2, SUM), (3, MAX)]
    assert finals == [(AVG, [1, 2]), (COUNT_ALL, [3]), (MAX, [4])]
    with pytest.raises(ValueError):
        split_requests([(0, 99)])


NB, NP = 3_000, 20_000


def join_data():
    import oracle as O
    bk = O.gen_keys(NB, np.int32, seed=7, groups=2_000)          # duplicate build keys
    pk = O.gen_keys(NP, np.int32, seed=8, groups=2_500)          # some probe keys absent
    return bk, pk


def oracle_join(bk, pk):
    import torch
    import oracle as O
    l, r = O.join_pairs(bk.numpy(), pk.numpy())
    return torch.from_numpy(l), torch.from_numpy(r)


def join_worker(rank, rdv, strategy, failures):
    import torch
    import torch.distributed as dist
    import oracle as O
    from eiger_b200.distributed import distributed_join
    try:
        dist.init_process_group("gloo", init_method=f"file://{rdv}", rank=rank, world_size=WORLD)
        bk, pk = join_data()
        blo, bhi = rank * NB // WORLD, (rank + 1) * NB // WORLD
        plo, phi = (rank * NP) // 3, ((rank + 1) * NP) // 3 if rank + 1 < WORLD else NP  # uneven shards
        b, p = distributed_join(torch.from_numpy(bk[blo:bhi].copy()), torch.from_numpy(pk[plo:phi].copy()), blo, plo,
                                strategy=strategy, local_join=oracle_join)
        # gather every rank's pairs on every rank and compare with the oracle
        n = torch.tensor([b.numel()], dtype=torch.int64)
        sizes = [torch.zeros_like(n) for _ in range(WORLD)]
        dist.all_gather(sizes, n)
        m = max(int(s.item()) for s in sizes)
        bb = torch.full((m,), -1, dtype=torch.int64)
        pp = torch.full((m,), -1, dtype=torch.int64)
        bb[: b.numel()], pp[: p.numel()] = b, p
        ab = [torch.empty_like(bb) for _ in range(WORLD)]
        ap = [torch.empty_like(pp) for _ in range(WORLD)]
        dist.all_gather(ab, bb)
        dist.all_gather(ap, pp)
        gb = torch.cat([x[: int(s.item())] for x, s in zip(ab, sizes)]).numpy()
        gp = torch.cat([x[: int(s.item())] for x, s in zip(ap, sizes)]).numpy()
        o = np.lexsort((gp, gb))
        el, er = O.join_pairs(bk, pk)
        assert np.array_equal(gb[o], el) and np.array_equal(gp[o], er)
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:
        failures.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


@pytest.mark.parametrize("strategy", ["broadcast", "shuffle"])
def test_two_rank_join_matches_single_oracle(strategy):
    ctx = mp.get_context("spawn")
    failures = ctx.SimpleQueue()
    with tempfile.TemporaryDirectory() as d:
        rdv = os.path.join(d, "rdv")
        procs = [ctx.Process(target=join_worker, args=(r, rdv, strategy, failures)) for r in range(WORLD)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        for p in procs:
            if p.is_alive():
                p.kill()
    msgs = []
    while not failures.empty():
        msgs.append(failures.get())
    assert not msgs, msgs
    assert all(p.exitcode == 0 for p in procs)
