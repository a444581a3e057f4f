"""Shared helpers for the GPU parity tests (device data <-> numpy, canonical
ordering, tolerance checks)."""
from __future__ import annotations

import numpy as np

FLOAT_RTOL = 1e-12   # float64 SUM / AVG: relative tolerance against the oracle
FLOAT32_RTOL = 1e-6  # float32 SUM: device accumulates in double, rounds once


def to_dev(a: np.ndarray):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.cuda()


def to_dev_raw(a: np.ndarray):
    """Upload any numpy array as raw bytes (for dtypes torch lacks)."""
    import torch
    b = np.ascontiguousarray(a).view(np.uint8)
    return torch.from_numpy(b.copy()).cuda()


def sort_by_key(cols: list[np.ndarray]) -> list[np.ndarray]:
    """Order result columns by the key column (column 0), ascending."""
    k = cols[0]
    if k.dtype.kind == "f":
        order = np.argsort(k, kind="stable")
    else:
        order = np.argsort(k, kind="stable")
    return [c[order] for c in cols]


def assert_columns_match(got: list[np.ndarray], exp: list[np.ndarray], float_cols_rtol=None):
    assert len(got) == len(exp), (len(got), len(exp))
    for i, (g, e) in enumerate(zip(got, exp)):
        assert g.dtype == e.dtype, (i, g.dtype, e.dtype)
        assert g.shape == e.shape, (i, g.shape, e.shape)
        if g.dtype.kind == "f":
            rtol = FLOAT32_RTOL if g.dtype == np.float32 else FLOAT_RTOL
            if float_cols_rtol is not None:
                rtol = float_cols_rtol
            both_nan = np.isnan(g) & np.isnan(e)
            diff = np.abs(g.astype(np.float64) - e.astype(np.float64))
            tol = rtol * np.maximum(np.abs(e.astype(np.float64)), 1e-300)
            bad = ~(both_nan | (diff <= tol) | (g == e))
            assert not bad.any(), (i, np.nonzero(bad)[0][:5], g[bad][:5], e[bad][:5])
        else:
            assert np.array_equal(g, e), (i, np.nonzero(g != e)[0][:5], g[g != e][:5], e[g != e][:5])
