"""Batched uneven string group-by pipelines (gx_batch_* C ABI).

Each instance holds an ARROW string column (ASCII keys drawn from a shared
dictionary), an int32 date column and an int64 fixed-point amount (scale 2).
A plan runs every instance's pipeline — dictionary-encode the strings, keep
rows with lo <= date < hi, group by the code with SUM(amount) and COUNT —
either as one persistent CUDA-graph launch (run) or as one operator sequence
per instance (run_per_instance).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np


def _gx():
    import eiger_b200 as gx
    return gx


def make_dictionary(size: int, seed: int, min_len: int = 8, max_len: int = 32):
    """`size` distinct ASCII strings with lengths uniform in [min_len, max_len]."""
    rng = np.random.default_rng(seed)
    seen, words = set(), []
    while len(words) < size:
        n = int(rng.integers(min_len, max_len + 1))
        w = bytes(rng.integers(33, 127, size=n, dtype=np.uint8))
        if w not in seen:
            seen.add(w)
            words.append(w)
    lens = np.array([len(w) for w in words], dtype=np.int64)
    offs = np.zeros(size + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    return np.frombuffer(b"".join(words), dtype=np.uint8).copy(), offs


@dataclass
class Instance:
    chars: object     # torch uint8 (device)
    offsets: object   # torch int64 (device), rows + 1
    date: object      # torch int32 (device)
    amount: object    # torch int64 (device)
    codes: object     # torch int32 (device): dictionary entry of each row (for checking)
    rows: int
    lo: int
    hi: int


def make_instances(count: int, seed: int, min_log2: int = 12, max_log2: int = 22, dict_size: int = 10_000,
                   date_span: int = 2557, keep: float = 0.4):
    """C5 instances: rows log-uniform in [2^min_log2, 2^max_log2]."""
    import torch
    gx = _gx()
    dchars, doffs = make_dictionary(dict_size, seed)
    d_dchars = torch.from_numpy(dchars).cuda()
    d_doffs = torch.from_numpy(doffs).cuda()
    dlens = d_doffs[1:] - d_doffs[:-1]
    rng = np.random.default_rng(seed + 1)
    out = []
    width = int(round(keep * date_span))
    for i in range(count):
        rows = int(2 ** rng.uniform(min_log2, max_log2))
        g = torch.Generator(device="cuda")
        g.manual_seed(int(seed * 7919 + i))
        codes = torch.randint(0, dict_size, (rows,), device="cuda", dtype=torch.int32, generator=g)
        offs = torch.zeros(rows + 1, dtype=torch.int64, device="cuda")
        torch.cumsum(dlens[codes.long()], 0, out=offs[1:])
        total = int(offs[-1].item())
        chars = torch.empty(max(total, 1), dtype=torch.uint8, device="cuda")
        gx.check(gx.lib.gx_generate_strings(d_dchars.data_ptr(), d_doffs.data_ptr(), dict_size, codes.data_ptr(),
                                            rows, offs.data_ptr(), chars.data_ptr(), None))
        date = torch.randint(0, date_span, (rows,), device="cuda", dtype=torch.int32, generator=g)
        amount = torch.randint(100, 10_000_000, (rows,), device="cuda", dtype=torch.int64, generator=g)
        lo = int(rng.integers(0, date_span - width + 1))
        out.append(Instance(chars, offs, date, amount, codes, rows, lo, lo + width))
    return out, (dchars, doffs)


class Plan:
    """A gx_batch_plan over a list of Instance objects."""

    def __init__(self, instances: list[Instance], max_distinct: int, stream=None):
        gx = _gx()
        self.instances = instances
        arr = (gx.BatchInstance * len(instances))()
        for i, it in enumerate(instances):
            arr[i] = gx.BatchInstance(it.chars.data_ptr(), it.offsets.data_ptr(), it.date.data_ptr(),
                                      it.amount.data_ptr(), it.rows, it.lo, it.hi)
        self._arr = arr
        self.handle = C.c_void_p()
        self.max_distinct = max_distinct
        gx.check(gx.lib.gx_batch_plan_create(arr, len(instances), max_distinct, gx._stream_ptr(stream),
                                             C.byref(self.handle)))

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value:
            _gx().lib.gx_batch_plan_free(self.handle)
            self.handle = C.c_void_p(0)

    def run(self, stream=None):
        gx = _gx()
        gx.check(gx.lib.gx_batch_run(self.handle, gx._stream_ptr(stream)))

    def run_per_instance(self, stream=None):
        gx = _gx()
        gx.check(gx.lib.gx_batch_run_per_instance(self.handle, gx._stream_ptr(stream)))

    def tuning(self) -> tuple[int, int]:
        gx = _gx()
        t, l = C.c_int32(), C.c_int32()
        gx.check(gx.lib.gx_batch_tuning(self.handle, C.byref(t), C.byref(l)))
        return t.value, l.value

    def results(self) -> list[dict]:
        """Per instance: {string bytes: (sum, count)} over groups with kept rows."""
        import torch
        gx = _gx()
        n = len(self.instances)
        res = (gx.BatchResult * n)()
        gx.check(gx.lib.gx_batch_results(self.handle, res))
        out = []
        for i, it in enumerate(self.instances):
            md = self.max_distinct
            s = np.empty(md, np.int64)
            c = np.empty(md, np.int64)
            f = np.empty(md, np.int64)
            for arr, ptr in ((s, res[i].sum), (c, res[i].count), (f, res[i].first_row)):
                gx.check(gx.lib.gx_copy(arr.ctypes.data, ptr, md * 8, None))
            chars = it.chars.cpu().numpy()
            offs = it.offsets.cpu().numpy()
            d = {}
            for code in np.nonzero(c > 0)[0]:
                r = f[code]
                d[bytes(chars[offs[r]:offs[r + 1]])] = (int(s[code]), int(c[code]))
            assert len(d) == res[i].num_groups
            out.append(d)
        return out
