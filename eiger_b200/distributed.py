"""Group-by over row shards held by several ranks (one process per GPU).

Each rank aggregates its own rows with the local engine, the partial
results are hash-partitioned by key and exchanged with one all-to-all, and
each rank merges the partials it received, so rank r ends up owning the
final groups whose key hashes to r.  Only partial aggregates cross the
interconnect (at most groups x ranks rows), never the input rows.

Merge rules (the aggregations are decomposable; the reference's aggregation
semantics are src/cuda/operators/groupby/agg_func.cuh:20-224):
    SUM -> SUM of partial sums        COUNT_ALL -> SUM of partial counts
    MIN -> MIN, MAX -> MAX, ANY -> ANY
    AVG -> SUM and COUNT_ALL partials, divided after the merge (float64,
           like groupby.cu:29-50).
Integer results are exact; a float64 SUM differs from the single-GPU order of
additions only by rounding.

The transport is torch.distributed (NCCL between GPUs; any backend with
all_to_all_single works, which is how the exchange is tested on CPU ranks).
"""
from __future__ import annotations

from typing import Callable, Sequence

SUM, MAX, MIN, AVG, ANY, COUNT_ALL = range(6)

_MERGE = {SUM: SUM, COUNT_ALL: SUM, MIN: MIN, MAX: MAX, ANY: ANY}


def split_requests(requests: Sequence[tuple[int, int]]):
    """Local requests, merge requests over the partial columns, and for each
    final output the partial columns (1-based: column 0 is the key) that make
    it: (kind, [partial column indexes])."""
    local, merge, finals = [], [], []
    for col, kind in requests:
        if kind == AVG:
            s, c = len(local), len(local) + 1
            local += [(col, SUM), (col, COUNT_ALL)]
            merge += [(s, SUM), (c, SUM)]
            finals.append((AVG, [1 + s, 1 + c]))
        elif kind in _MERGE:
            i = len(local)
            local.append((col, kind))
            merge.append((i, _MERGE[kind]))
            finals.append((kind, [1 + i]))
        else:
            raise ValueError(f"aggregation kind {kind} cannot be merged across ranks")
    return local, merge, finals


def destination(keys, world: int):
    """Owner rank of each key: a multiplicative hash of the key bits."""
    import torch
    k = keys.view(torch.int32).to(torch.int64) if keys.element_size() == 4 else keys.view(torch.int64)
    h = (k * -7046029254386353131) >> 17  # 0x9E3779B97F4A7C15 as int64; wraps like uint64
    return (h & 0x7FFFFFFF) % world


def _as_wire(t):
    """Same bytes as a dtype every backend can move (int32 / int64 / float64)."""
    import torch
    if t.dtype in (torch.int32, torch.int64, torch.float64, torch.float32):
        return t, t.dtype
    w = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[t.element_size()]
    return t.view(w), t.dtype


def exchange(columns: list, dest, world: int, group=None) -> list:
    """Send row i of every column to rank dest[i]; returns the received rows."""
    import torch
    import torch.distributed as dist
    order = torch.argsort(dest, stable=True)
    send = torch.bincount(dest, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    send_l, recv_l = send.tolist(), recv.tolist()
    out = []
    for c in columns:
        w, dt = _as_wire(c[order].contiguous())
        r = torch.empty(sum(recv_l), dtype=w.dtype, device=w.device)
        dist.all_to_all_single(r, w, recv_l, send_l, group=group)
        out.append(r.view(dt) if dt != w.dtype else r)
    return out


def _gx_local(keys, vals, requests):
    import eiger_b200 as gx
    t = gx.groupby([keys], list(vals), requests, gx.make_hint(gx.AUTO_ALGO))
    return [t.to_torch(i) for i in range(t.num_columns)]


def distributed_groupby(keys, vals: Sequence, requests: Sequence[tuple[int, int]],
                        local_groupby: Callable | None = None, group=None) -> list:
    """This rank's share of the global group-by of the row shards on all ranks.

    Returns [key, one column per request] for the keys this rank owns.
    `local_groupby(keys, vals, requests) -> [key, agg...]` defaults to the
    library's engine on the GPU.
    """
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    run = local_groupby or _gx_local
    local, merge, finals = split_requests(requests)
    part = run(keys, vals, local)
    dest = destination(part[0], world)
    got = exchange(part, dest, world, group)
    merged = run(got[0], got[1:], merge)
    out = [merged[0]]
    for kind, cols in finals:
        if kind == AVG:
            s, c = merged[cols[0]], merged[cols[1]]
            out.append(s.to(torch.float64) / c.to(torch.float64))
        else:
            out.append(merged[cols[0]])
    return out


# ---------------------------------------------------------------------------
# Inner equi-join over row shards.
# ---------------------------------------------------------------------------
def _all_gather_uneven(t, world: int, group=None):
    """Concatenation of every rank's 1-D tensor t (shards of any length)."""
    import torch
    import torch.distributed as dist
    n = torch.tensor([t.numel()], dtype=torch.int64, device=t.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    w, dt = _as_wire(t.contiguous())
    m = max(sizes) if sizes else 0
    pad = torch.zeros(m, dtype=w.dtype, device=w.device)
    pad[: w.numel()] = w
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    out = torch.cat([p[:s] for p, s in zip(parts, sizes)])
    return out.view(dt) if dt != w.dtype else out


def _gx_join(build_keys, probe_keys):
    import eiger_b200 as gx
    t = gx.inner_eq_join_rowids(build_keys, probe_keys, gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR))
    return t.to_torch(0), t.to_torch(1)


def distributed_join(build_keys, probe_keys, build_base: int, probe_base: int, strategy: str = "broadcast",
                     local_join: Callable | None = None, group=None):
    """This rank's share of the inner equi-join of the build and probe row
    shards held by all ranks.  Row i of this rank's build (probe) shard has
    global row id build_base + i (probe_base + i).  Returns the matched
    (global build row, global probe row) pairs found on this rank; the
    union over ranks is the join of all rows, each pair exactly once.

    strategy "broadcast": every rank gathers the whole build side (keys and
    row ids, 12 B per build row for int32 keys) and probes its own probe
    shard; nothing of the probe side moves.  Suits a small build side (the
    2^24-row build of a 2^28-row probe moves 200 MB to each GPU).
    strategy "shuffle": both sides are hash-partitioned by key with one
    all-to-all each, then joined locally; every row crosses the interconnect
    at most once.  Suits two large sides.

    `local_join(build_keys, probe_keys) -> (build_rows, probe_rows)` (local
    row positions) defaults to the library's join on the GPU.
    """
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    run = local_join or _gx_join
    dev = build_keys.device
    brow = torch.arange(build_keys.numel(), dtype=torch.int64, device=dev) + build_base
    prow = torch.arange(probe_keys.numel(), dtype=torch.int64, device=dev) + probe_base
    if strategy == "broadcast":
        bk = _all_gather_uneven(build_keys, world, group)
        br = _all_gather_uneven(brow, world, group)
        pk, pr = probe_keys, prow
    elif strategy == "shuffle":
        bk, br = exchange([build_keys, brow], destination(build_keys, world), world, group)
        pk, pr = exchange([probe_keys, prow], destination(probe_keys, world), world, group)
    else:
        raise ValueError(f"unknown join strategy {strategy!r}")
    l, r = run(bk, pk)
    return br[l.long()], pr[r.long()]
