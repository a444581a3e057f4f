"""CPU restatement of the batched string pipeline — TEST INFRASTRUCTURE ONLY.

Per instance: keep rows with lo <= date < hi, group them by the bytes of
their string key, SUM(amount) and COUNT (the dictionary-encode -> select ->
group-by pipeline of the batched engine, checked on the strings themselves).
"""
from __future__ import annotations

import numpy as np


def string_groupby(chars: np.ndarray, offsets: np.ndarray, date: np.ndarray, amount: np.ndarray, lo: int,
                   hi: int) -> dict:
    keep = np.nonzero((date >= lo) & (date < hi))[0]
    out: dict = {}
    raw = chars.tobytes()
    for r in keep:
        k = raw[offsets[r]:offsets[r + 1]]
        s, c = out.get(k, (0, 0))
        out[k] = (s + int(amount[r]), c + 1)
    return out
