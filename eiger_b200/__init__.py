"""eiger_b200 — B200-native relational operator core (Python binding).

Thin ctypes binding over the C ABI in include/gx.h (libgx.so, built for
sm_100a by eiger_b200/build.py).  The functions mirror the reference's
operator API (gamax::groupby::groupby, gamax::join::inner_eq_join,
gamax::sort::*, gamax::partition::*, gamax::compress::*), taking device
columns as torch tensors and returning owned result tables.

There is no CPU fallback: importing the package loads libgx.so and raises
if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

_PKG = Path(__file__).resolve().parent
_LIB_PATH = _PKG / "libgx.so"

# ---------------------------------------------------------------------------
# Enumerations (include/gx.h; same order as gamax::type_id and friends)
# ---------------------------------------------------------------------------
EMPTY, INT8, INT16, INT32, INT64, BOOL8, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64, STRING = range(13)
SUM, MAX, MIN, AVG, ANY, COUNT_ALL = range(6)
AUTO_ALGO, HASH, SORT, SORT_OPT, SORT_GFUR, PARTITION, PARTITION_GFUR = range(7)
JOIN_AUTO, JOIN_HASH, JOIN_SORT, JOIN_PARTITION = range(4)
MAT_AUTO, MAT_GFUR, MAT_GFTR, MAT_INDEX_CLUSTER = range(4)
SORTED_BUILD, SORT_MERGE = 0, 1
ASCENDING, DESCENDING = 0, 1
SELECT_HEURISTIC, SELECT_LEARNED = 0, 1
CMP_LT, CMP_LE, CMP_GT, CMP_GE, CMP_EQ, CMP_NE, CMP_BETWEEN = range(7)
COMBINE_AND, COMBINE_OR = 0, 1
DIST_UNIFORM, DIST_CYCLIC, DIST_ZIPF, DIST_SEQUENCE, DIST_ZIPF_APPROX = range(5)

STATUS = {0: "GX_OK", 1: "GX_EINVAL", 2: "GX_ENOMEM", 3: "GX_ECUDA", 4: "GX_EOVERFLOW",
          5: "GX_ETIMEOUT", 6: "GX_EUNSUPPORTED"}

_NP = {INT8: np.int8, INT16: np.int16, INT32: np.int32, INT64: np.int64, BOOL8: np.bool_,
       UINT8: np.uint8, UINT16: np.uint16, UINT32: np.uint32, UINT64: np.uint64,
       FLOAT32: np.float32, FLOAT64: np.float64}
_NP_TO_GX = {np.dtype(v): k for k, v in _NP.items()}


def size_of(t: int) -> int:
    return np.dtype(_NP[t]).itemsize if t in _NP else 0


class GxError(RuntimeError):
    """A non-GX_OK status from the library (message from gx_last_error_message)."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


# ---------------------------------------------------------------------------
# ctypes structures
# ---------------------------------------------------------------------------
class ColumnView(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_int64), ("type", C.c_int32), ("offset", C.c_int64)]


class StringColumns(C.Structure):
    _fields_ = [("chars", C.c_void_p), ("offsets", C.c_void_p)]


class TableView(C.Structure):
    _fields_ = [("columns", C.POINTER(ColumnView)), ("num_columns", C.c_int64)]


class OwnedColumn(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_int64), ("type", C.c_int32), ("capacity_bytes", C.c_int64)]


class AggRequest(C.Structure):
    _fields_ = [("column_index", C.c_int64), ("agg_kind", C.c_int32)]


class GroupbyHint(C.Structure):
    _fields_ = [("groups_upper_bound", C.c_int64), ("zero_based_ids", C.c_int32), ("optimize_sort", C.c_int32),
                ("groupby_algo", C.c_int32), ("agg_count", C.c_int32), ("enable_skf", C.c_int32),
                ("allow_hash_fallback", C.c_int32), ("selector", C.c_int32), ("radix_bits", C.c_int32),
                ("load_factor_pct", C.c_int32), ("reserved", C.c_int32)]


class JoinHint(C.Structure):
    _fields_ = [("sorted_left", C.c_int32), ("sorted_right", C.c_int32), ("unique_left", C.c_int32),
                ("unique_right", C.c_int32), ("max_out", C.c_int64), ("join_algo", C.c_int32),
                ("mat_algo", C.c_int32), ("sort_mode", C.c_int32), ("reserved", C.c_int32)]


class GenSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("stream_id", C.c_uint64), ("dist", C.c_int32), ("scatter", C.c_int32),
                ("groups", C.c_int64), ("zipf_s", C.c_double), ("zipf_cdf", C.c_void_p), ("lo", C.c_int64),
                ("hi", C.c_int64), ("miss_frac", C.c_double)]


class Predicate(C.Structure):
    _fields_ = [("column_index", C.c_int64), ("op", C.c_int32), ("reserved", C.c_int32), ("lo_i", C.c_int64),
                ("hi_i", C.c_int64), ("lo_f", C.c_double), ("hi_f", C.c_double)]


class BatchInstance(C.Structure):
    _fields_ = [("chars", C.c_void_p), ("offsets", C.c_void_p), ("date", C.c_void_p), ("amount", C.c_void_p),
                ("rows", C.c_int64), ("date_lo", C.c_int32), ("date_hi", C.c_int32)]


class BatchResult(C.Structure):
    _fields_ = [("num_groups", C.c_int64), ("sum", C.c_void_p), ("count", C.c_void_p), ("first_row", C.c_void_p)]


# ---------------------------------------------------------------------------
# Library loading
# ---------------------------------------------------------------------------
def _load() -> C.CDLL:
    path = os.environ.get("GX_LIB", str(_LIB_PATH))
    if not Path(path).exists():
        raise ImportError(f"libgx.so not found at {path}; build it with `python eiger_b200/build.py`")
    lib = C.CDLL(path)
    vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    tv, cv = C.POINTER(TableView), ColumnView
    oc = C.POINTER(OwnedColumn)
    sig = {
        "gx_last_error_message": ([], C.c_char_p),
        "gx_version": ([], C.c_char_p),
        "gx_kernel_launch_count": ([], i64),
        "gx_table_num_columns": ([vp], i64),
        "gx_table_num_rows": ([vp], i64),
        "gx_table_column": ([vp, i64, C.POINTER(ColumnView)], i32),
        "gx_table_release_column": ([vp, i64, oc], i32),
        "gx_table_free": ([vp], None),
        "gx_malloc": ([C.POINTER(vp), C.c_size_t, vp], i32),
        "gx_free": ([vp, vp], i32),
        "gx_mem_stats": ([C.POINTER(i64), C.POINTER(i64)], i32),
        "gx_mem_reset_peak": ([], i32),
        "gx_copy": ([vp, vp, C.c_size_t, vp], i32),
        "gx_stream_sync": ([vp], i32),
        "gx_groupby_hint_init": ([C.POINTER(GroupbyHint)], None),
        "gx_join_hint_init": ([C.POINTER(JoinHint)], None),
        "gx_agg_output_type": ([i32, i32], i32),
        "gx_inner_eq_join": ([tv, tv, C.POINTER(JoinHint), vp, C.POINTER(vp)], i32),
        "gx_inner_eq_join_rowids": ([cv, cv, C.POINTER(JoinHint), vp, C.POINTER(vp)], i32),
        "gx_sort_temp_bytes": ([i64, i32, i32, C.POINTER(C.c_size_t)], i32),
        "gx_sort_column_pair": ([cv, cv, i32, i32, i32, vp, C.c_size_t, vp, oc, oc], i32),
        "gx_sort_column": ([cv, i32, i32, i32, vp, C.c_size_t, vp, oc], i32),
        "gx_argsort": ([cv, i32, i32, i32, vp, C.c_size_t, vp, oc, oc], i32),
        "gx_partition_column_pair": ([cv, cv, i32, i32, vp, C.c_size_t, vp, oc, oc], i32),
        "gx_partition_column": ([cv, i32, i32, vp, C.c_size_t, vp, oc], i32),
        "gx_arg_partition": ([cv, i32, i32, vp, C.c_size_t, vp, oc, oc], i32),
        "gx_compute_partition_offsets": ([cv, i32, i32, vp, oc], i32),
        "gx_dictionary_encode": ([cv, i32, i64, f64, vp, oc, C.POINTER(i64)], i32),
        "gx_dictionary_encode_with_order": ([cv, i32, i64, f64, vp, oc, C.POINTER(i64)], i32),
        "gx_dictionary_encode_with_dict": ([cv, cv, i32, vp, oc], i32),
        "gx_dictionary_encode_strings": ([cv, i64, vp, oc, C.POINTER(i64)], i32),
        "gx_compute_ndv_approx": ([cv, vp, C.POINTER(i64)], i32),
        "gx_compute_min_max": ([cv, vp, vp, vp], i32),
        "gx_zipf_cdf_host": ([i64, f64, vp], i32),
        "gx_generate_keys": ([cv, C.POINTER(GenSpec), vp], i32),
        "gx_generate_values": ([cv, C.POINTER(GenSpec), vp], i32),
        "gx_generate_permutation": ([cv, C.c_uint64, i64, vp], i32),
        "gx_generate_strings": ([vp, vp, i64, vp, i64, vp, vp, vp], i32),
        "gx_fill_sequence": ([cv, i64, i64, vp], i32),
        "gx_profile_enable": ([i32], None),
        "gx_profile_reset": ([], None),
        "gx_profile_read": ([C.c_char_p, C.POINTER(C.c_double), C.POINTER(i64)], i32),
        "gx_selector_features": ([cv, vp, vp], i32),
        "gx_selector_plan_features": ([tv, C.POINTER(AggRequest), i32, i32, vp], i32),
        "gx_selector_param_count": ([], i64),
        "gx_selector_load": ([vp, vp, vp], i32),
        "gx_selector_set_plan_support": ([vp, i32, C.c_float], i32),
        "gx_selector_predict": ([vp, i32, vp], i32),
        "gx_mlp_forward": ([vp, vp, i32, vp, vp], i32),
        "gx_mlp_forward_backward": ([vp, vp, vp, vp, i32, vp, vp, vp], i32),
        "gx_mlp_adam_step": ([vp, vp, vp, vp, vp, i32, C.c_float, vp], i32),
        "gx_batch_plan_create": ([C.POINTER(BatchInstance), i32, i64, vp, C.POINTER(vp)], i32),
        "gx_batch_run": ([vp, vp], i32),
        "gx_batch_run_per_instance": ([vp, vp], i32),
        "gx_batch_results": ([vp, C.POINTER(BatchResult)], i32),
        "gx_batch_tuning": ([vp, C.POINTER(i32), C.POINTER(i32)], i32),
        "gx_batch_plan_free": ([vp], None),
        "gx_multikey_compress": ([tv, i32, vp, oc, C.POINTER(i32)], i32),
        "gx_gather": ([cv, cv, vp, oc], i32),
        "gx_select_to_bitmask": ([tv, C.POINTER(Predicate), i32, i32, vp, oc], i32),
        "gx_select": ([tv, C.POINTER(Predicate), i32, i32, vp, C.POINTER(vp)], i32),
        "gx_compact": ([tv, cv, vp, C.POINTER(vp)], i32),
        "gx_count_nonzero": ([cv, vp, C.POINTER(i64)], i32),
    }
    for name in ("gx_groupby", "gx_groupby_hash", "gx_groupby_sort", "gx_groupby_sort_gfur",
                 "gx_groupby_partition", "gx_groupby_partition_gfur"):
        sig[name] = ([tv, tv, C.POINTER(AggRequest), i32, C.POINTER(GroupbyHint), vp, C.POINTER(vp)], i32)
    for name in ("gx_distinct_hash", "gx_distinct_sort"):
        sig[name] = ([tv, C.POINTER(GroupbyHint), vp, C.POINTER(vp)], i32)
    sig["gx_aggregate"] = ([tv, C.POINTER(AggRequest), i32, vp, C.POINTER(vp)], i32)
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()

def check(status: int) -> None:
    if status != 0:
        raise GxError(status, lib.gx_last_error_message().decode(errors="replace"))


def last_error() -> str:
    return lib.gx_last_error_message().decode(errors="replace")


def kernel_launches() -> int:
    return int(lib.gx_kernel_launch_count())


# ---------------------------------------------------------------------------
# torch helpers (imported lazily so the CPU test suite stays light)
# ---------------------------------------------------------------------------
def _torch():
    import torch
    return torch


def gx_type_of(t) -> int:
    torch = _torch()
    m = {torch.int8: INT8, torch.int16: INT16, torch.int32: INT32, torch.int64: INT64, torch.bool: BOOL8,
         torch.uint8: UINT8, torch.float32: FLOAT32, torch.float64: FLOAT64}
    for name, code in (("uint16", UINT16), ("uint32", UINT32), ("uint64", UINT64)):
        if hasattr(torch, name):
            m[getattr(torch, name)] = code
    return m[t.dtype]


def torch_dtype(t: int):
    torch = _torch()
    m = {INT8: torch.int8, INT16: torch.int16, INT32: torch.int32, INT64: torch.int64, BOOL8: torch.bool,
         UINT8: torch.uint8, FLOAT32: torch.float32, FLOAT64: torch.float64,
         UINT16: getattr(torch, "uint16", torch.int16), UINT32: getattr(torch, "uint32", torch.int32),
         UINT64: getattr(torch, "uint64", torch.int64)}
    return m[t]


def view(t, gx_type: int | None = None, offset: int = 0) -> ColumnView:
    """Column view over a contiguous CUDA tensor (optionally reinterpreted)."""
    assert t.is_cuda and t.is_contiguous(), "device, contiguous tensor required"
    ty = gx_type if gx_type is not None else gx_type_of(t)
    n = t.numel() * t.element_size() // max(size_of(ty), 1)
    return ColumnView(t.data_ptr(), n - offset, ty, offset)


class StringColumn:
    """A device STRING column in the ARROW layout: `chars` (uint8 tensor) and
    `offsets` (int64 tensor, rows + 1 entries); `row_offset` skips rows like
    a column view's offset.  Usable wherever a key column is accepted."""

    def __init__(self, chars, offsets, rows: int | None = None, row_offset: int = 0):
        self.chars, self.offsets = chars, offsets
        self.row_offset = row_offset
        self.rows = (offsets.numel() - 1 - row_offset) if rows is None else rows
        self._sc = StringColumns(chars.data_ptr(), offsets.data_ptr())

    def view(self) -> ColumnView:
        return ColumnView(C.cast(C.pointer(self._sc), C.c_void_p), self.rows, STRING, self.row_offset)

    @staticmethod
    def from_list(strs: Sequence[bytes]) -> "StringColumn":
        """Uploads a list of byte strings."""
        torch = _torch()
        lens = np.array([len(x) for x in strs], dtype=np.int64)
        off = np.zeros(len(strs) + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        chars = np.frombuffer(b"".join(strs), dtype=np.uint8) if off[-1] else np.zeros(1, np.uint8)
        return StringColumn(torch.from_numpy(chars.copy()).cuda(), torch.from_numpy(off).cuda(), len(strs))


def _column_view(c) -> ColumnView:
    if isinstance(c, ColumnView):
        return c
    if isinstance(c, StringColumn):
        return c.view()
    return view(c)


def table_view(cols: Sequence) -> tuple[TableView, object]:
    arr = (ColumnView * max(len(cols), 1))()
    for i, c in enumerate(cols):
        arr[i] = _column_view(c)
    return TableView(arr, len(cols)), (arr, list(cols))


def strings_from_device(v: ColumnView) -> np.ndarray:
    """Copies a STRING column view (host gx_string_columns -> device
    chars / offsets) to a numpy object array of bytes."""
    n = v.size
    if n == 0:
        return np.array([], dtype=object)
    sc = C.cast(v.data, C.POINTER(StringColumns)).contents
    off = np.empty(n + 1, dtype=np.int64)
    check(lib.gx_copy(off.ctypes.data, sc.offsets + 8 * v.offset, off.nbytes, None))
    chars = np.empty(max(int(off[-1] - off[0]), 1), dtype=np.uint8)
    if off[-1] > off[0]:
        check(lib.gx_copy(chars.ctypes.data, sc.chars + int(off[0]), int(off[-1] - off[0]), None))
    b = chars.tobytes()
    base = int(off[0])
    out = np.empty(n, dtype=object)
    for i in range(n):
        out[i] = b[off[i] - base:off[i + 1] - base]
    return out


def _stream_ptr(stream) -> int | None:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    return stream if isinstance(stream, int) else stream.cuda_stream


class Table:
    """An owned result table (gx_table*)."""

    def __init__(self, handle: int):
        self.handle = C.c_void_p(handle)

    def __del__(self):
        # At interpreter exit the module globals may already be gone; the
        # process teardown releases the device memory then.
        if getattr(self, "handle", None) and self.handle.value and lib is not None:
            lib.gx_table_free(self.handle)
            self.handle = C.c_void_p(0)

    @property
    def num_columns(self) -> int:
        return int(lib.gx_table_num_columns(self.handle))

    @property
    def num_rows(self) -> int:
        return int(lib.gx_table_num_rows(self.handle))

    def column(self, i: int) -> ColumnView:
        v = ColumnView()
        check(lib.gx_table_column(self.handle, i, C.byref(v)))
        return v

    def type(self, i: int) -> int:
        return self.column(i).type

    def to_numpy(self, i: int) -> np.ndarray:
        v = self.column(i)
        if v.type == STRING:
            return strings_from_device(v)
        out = np.empty(v.size, dtype=_NP[v.type])
        if v.size:
            check(lib.gx_copy(out.ctypes.data, v.data, out.nbytes, None))
        return out

    def to_torch(self, i: int):
        torch = _torch()
        v = self.column(i)
        out = torch.empty(v.size, dtype=torch_dtype(v.type), device="cuda")
        if v.size:
            check(lib.gx_copy(out.data_ptr(), v.data, v.size * size_of(v.type), None))
        return out

    def numpy_columns(self) -> list[np.ndarray]:
        return [self.to_numpy(i) for i in range(self.num_columns)]


def owned_to_torch(oc: OwnedColumn, stream=None):
    """Copy an owned column into a torch tensor and free the library buffer."""
    torch = _torch()
    out = torch.empty(oc.size, dtype=torch_dtype(oc.type), device="cuda")
    if oc.size:
        check(lib.gx_copy(out.data_ptr(), oc.data, oc.size * size_of(oc.type), None))
    if oc.data:
        check(lib.gx_free(oc.data, None))
    return out


def make_hint(algo: int = AUTO_ALGO, groups_upper_bound: int | None = None, **kw) -> GroupbyHint:
    h = GroupbyHint()
    lib.gx_groupby_hint_init(C.byref(h))
    h.groupby_algo = algo
    if groups_upper_bound is not None:
        h.groups_upper_bound = groups_upper_bound
    for k, v in kw.items():
        setattr(h, k, v)
    return h


_GROUPBY_FN = {None: "gx_groupby", HASH: "gx_groupby_hash", SORT: "gx_groupby_sort",
               SORT_GFUR: "gx_groupby_sort_gfur", PARTITION: "gx_groupby_partition",
               PARTITION_GFUR: "gx_groupby_partition_gfur"}


def groupby(keys: Sequence, vals: Sequence, requests: Iterable[tuple[int, int]], hint: GroupbyHint | None = None,
            stream=None, entry: int | None = None) -> Table:
    """gamax::groupby::groupby: returns [key, aggregates in request order (+count)]."""
    hint = hint if hint is not None else make_hint()
    ktv, _k = table_view(keys)
    vtv, _v = table_view(vals)
    reqs = list(requests)
    arr = (AggRequest * max(len(reqs), 1))(*[AggRequest(c, k) for c, k in reqs])
    out = C.c_void_p()
    fn = getattr(lib, _GROUPBY_FN[entry])
    check(fn(C.byref(ktv), C.byref(vtv), arr, len(reqs), C.byref(hint), _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def distinct(keys: Sequence, hint: GroupbyHint | None = None, algo: int = HASH, stream=None) -> Table:
    """hash::distinct / sort::distinct: one row per distinct key row."""
    hint = hint if hint is not None else make_hint(algo)
    ktv, _k = table_view(keys)
    out = C.c_void_p()
    fn = lib.gx_distinct_sort if algo in (SORT, SORT_OPT, SORT_GFUR) else lib.gx_distinct_hash
    check(fn(C.byref(ktv), C.byref(hint), _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def aggregate(cols: Sequence, requests: Iterable[tuple[int, int]], stream=None) -> Table:
    """groupby::aggregate::aggregate: one-row table of whole-column aggregates."""
    tv, _t = table_view(cols)
    reqs = list(requests)
    arr = (AggRequest * max(len(reqs), 1))(*[AggRequest(c, k) for c, k in reqs])
    out = C.c_void_p()
    check(lib.gx_aggregate(C.byref(tv), arr, len(reqs), _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def predicate(column: int, op: int, lo=0, hi=0) -> Predicate:
    """column (op) literal; BETWEEN keeps lo <= x < hi.  The literal is used
    as an integer for integer columns and as a double for float columns."""
    def i64(x):  # uint64 literals above 2^63 travel as their two's-complement bits
        x = int(x)
        return x - (1 << 64) if x >= (1 << 63) else x

    p = Predicate()
    p.column_index, p.op = column, op
    p.lo_f, p.hi_f = float(lo), float(hi)
    p.lo_i, p.hi_i = i64(lo), i64(hi)
    return p


def _preds(preds):
    return (Predicate * max(len(preds), 1))(*preds), len(preds)


def select_to_bitmask(cols: Sequence, preds: Sequence[Predicate], combine=COMBINE_AND, stream=None):
    tv, _t = table_view(cols)
    arr, n = _preds(preds)
    o = OwnedColumn()
    check(lib.gx_select_to_bitmask(C.byref(tv), arr, n, combine, _stream_ptr(stream), C.byref(o)))
    return owned_to_torch(o)


def select(cols: Sequence, preds: Sequence[Predicate], combine=COMBINE_AND, stream=None) -> Table:
    tv, _t = table_view(cols)
    arr, n = _preds(preds)
    out = C.c_void_p()
    check(lib.gx_select(C.byref(tv), arr, n, combine, _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def compact(cols: Sequence, mask, stream=None) -> Table:
    tv, _t = table_view(cols)
    out = C.c_void_p()
    check(lib.gx_compact(C.byref(tv), view(mask, BOOL8 if mask.element_size() == 1 else None),
                         _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def count_nonzero(col, stream=None) -> int:
    c = C.c_int64()
    check(lib.gx_count_nonzero(view(col), _stream_ptr(stream), C.byref(c)))
    return int(c.value)


def make_join_hint(join_algo=JOIN_SORT, mat_algo=MAT_GFUR, **kw) -> JoinHint:
    h = JoinHint()
    lib.gx_join_hint_init(C.byref(h))
    h.join_algo, h.mat_algo = join_algo, mat_algo
    for k, v in kw.items():
        setattr(h, k, v)
    return h


def inner_eq_join(left: Sequence, right: Sequence, hint: JoinHint | None = None, stream=None) -> Table:
    """gamax::join::inner_eq_join: [key, left payloads..., right payloads...]."""
    hint = hint if hint is not None else make_join_hint()
    ltv, _l = table_view(left)
    rtv, _r = table_view(right)
    out = C.c_void_p()
    check(lib.gx_inner_eq_join(C.byref(ltv), C.byref(rtv), C.byref(hint), _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def inner_eq_join_rowids(lkey, rkey, hint: JoinHint | None = None, stream=None) -> Table:
    hint = hint if hint is not None else make_join_hint()
    out = C.c_void_p()
    lv = lkey if isinstance(lkey, ColumnView) else view(lkey)
    rv = rkey if isinstance(rkey, ColumnView) else view(rkey)
    check(lib.gx_inner_eq_join_rowids(lv, rv, C.byref(hint), _stream_ptr(stream), C.byref(out)))
    return Table(out.value)


def sort_column_pair(key, val, begin_bit=0, end_bit=-1, order=ASCENDING, stream=None):
    ko, vo = OwnedColumn(), OwnedColumn()
    check(lib.gx_sort_column_pair(view(key), view(val), begin_bit, end_bit, order, None, 0, _stream_ptr(stream),
                                  C.byref(ko), C.byref(vo)))
    return owned_to_torch(ko), owned_to_torch(vo)


def sort_column(col, begin_bit=0, end_bit=-1, order=ASCENDING, stream=None):
    ko = OwnedColumn()
    check(lib.gx_sort_column(view(col), begin_bit, end_bit, order, None, 0, _stream_ptr(stream), C.byref(ko)))
    return owned_to_torch(ko)


def argsort(col, begin_bit=0, end_bit=-1, order=ASCENDING, stream=None):
    ko, io = OwnedColumn(), OwnedColumn()
    check(lib.gx_argsort(view(col), begin_bit, end_bit, order, None, 0, _stream_ptr(stream), C.byref(ko),
                         C.byref(io)))
    return owned_to_torch(ko), owned_to_torch(io)


def partition_column_pair(key, val, begin_bit, end_bit, stream=None):
    ko, vo = OwnedColumn(), OwnedColumn()
    check(lib.gx_partition_column_pair(view(key), view(val), begin_bit, end_bit, None, 0, _stream_ptr(stream),
                                       C.byref(ko), C.byref(vo)))
    return owned_to_torch(ko), owned_to_torch(vo)


def partition_column(col, begin_bit, end_bit, stream=None):
    ko = OwnedColumn()
    check(lib.gx_partition_column(view(col), begin_bit, end_bit, None, 0, _stream_ptr(stream), C.byref(ko)))
    return owned_to_torch(ko)


def arg_partition(col, begin_bit, end_bit, stream=None):
    ko, io = OwnedColumn(), OwnedColumn()
    check(lib.gx_arg_partition(view(col), begin_bit, end_bit, None, 0, _stream_ptr(stream), C.byref(ko),
                               C.byref(io)))
    return owned_to_torch(ko), owned_to_torch(io)


def compute_partition_offsets(col, begin_bit, end_bit, stream=None):
    o = OwnedColumn()
    check(lib.gx_compute_partition_offsets(view(col), begin_bit, end_bit, _stream_ptr(stream), C.byref(o)))
    return owned_to_torch(o)


def dictionary_encode(col, encode_type=INT32, size_hint=0, load_factor=0.25, ordered=False, stream=None):
    o, nd = OwnedColumn(), C.c_int64()
    fn = lib.gx_dictionary_encode_with_order if ordered else lib.gx_dictionary_encode
    check(fn(view(col), encode_type, size_hint, load_factor, _stream_ptr(stream), C.byref(o), C.byref(nd)))
    return owned_to_torch(o), int(nd.value)


def dictionary_encode_with_dict(col, dictionary, encode_type=INT32, stream=None):
    o = OwnedColumn()
    check(lib.gx_dictionary_encode_with_dict(view(col), view(dictionary), encode_type, _stream_ptr(stream),
                                             C.byref(o)))
    return owned_to_torch(o)


def dictionary_encode_strings(chars, offsets, rows: int | None = None, row_offset: int = 0, size_hint: int = 0,
                              stream=None):
    """Hash-encode an ARROW string column (device chars + int64 offsets):
    returns (int32 codes, NDV)."""
    n = (offsets.numel() - 1 - row_offset) if rows is None else rows
    sc = StringColumns(chars.data_ptr(), offsets.data_ptr())
    v = ColumnView(C.cast(C.pointer(sc), C.c_void_p), n, STRING, row_offset)
    o, nd = OwnedColumn(), C.c_int64()
    check(lib.gx_dictionary_encode_strings(v, size_hint, _stream_ptr(stream), C.byref(o), C.byref(nd)))
    return owned_to_torch(o), nd.value


def multikey_compress(keys: Sequence, max_bits: int = 64, stream=None):
    """Smart key fusion of integral key columns: (UINT64 tensor, bits used),
    or None when the keys cannot be fused (compress::multikey_compress)."""
    tv, _keep = table_view(keys)
    o, bits = OwnedColumn(), C.c_int32()
    st = lib.gx_multikey_compress(C.byref(tv), max_bits, _stream_ptr(stream), C.byref(o), C.byref(bits))
    if st == 6:  # GX_EUNSUPPORTED: not compressible
        return None
    check(st)
    return owned_to_torch(o), bits.value


def gather(gather_map, col, stream=None):
    """out[i] = col[gather_map[i]] (util::device::gather); STRING columns
    (StringColumn) come back as a numpy object array of bytes."""
    o = OwnedColumn()
    check(lib.gx_gather(view(gather_map), _column_view(col), _stream_ptr(stream), C.byref(o)))
    if o.type != STRING:
        return owned_to_torch(o)
    n = o.size
    off = np.empty(n + 1, dtype=np.int64)
    check(lib.gx_copy(off.ctypes.data, o.data, off.nbytes, None))
    chars = np.empty(max(int(off[-1]), 1), dtype=np.uint8)
    if off[-1]:
        check(lib.gx_copy(chars.ctypes.data, o.data + 8 * (n + 1), int(off[-1]), None))
    check(lib.gx_free(o.data, None))
    b = chars.tobytes()
    out = np.empty(n, dtype=object)
    for i in range(n):
        out[i] = b[off[i]:off[i + 1]]
    return out


def compute_ndv_approx(col, stream=None) -> int:
    """HyperLogLog distinct-count estimate of a device column (a tensor or a
    ColumnView)."""
    nd = C.c_int64()
    check(lib.gx_compute_ndv_approx(_column_view(col), _stream_ptr(stream), C.byref(nd)))
    return int(nd.value)


# ---------------------------------------------------------------------------
# Generators
# ---------------------------------------------------------------------------
def gen_spec(seed=42, stream_id=0, dist=DIST_UNIFORM, scatter=0, groups=1, zipf_s=0.0, zipf_cdf=None, lo=0,
             hi=1, miss_frac=0.0) -> GenSpec:
    return GenSpec(seed, stream_id, dist, scatter, groups, zipf_s, zipf_cdf or 0, lo, hi, miss_frac)


def zipf_cdf(groups: int, s: float) -> np.ndarray:
    out = np.empty(groups, dtype=np.float64)
    check(lib.gx_zipf_cdf_host(groups, s, out.ctypes.data))
    return out


def generate_keys(out, spec: GenSpec, stream=None):
    check(lib.gx_generate_keys(view(out), C.byref(spec), _stream_ptr(stream)))
    return out


def generate_values(out, spec: GenSpec, stream=None):
    check(lib.gx_generate_values(view(out), C.byref(spec), _stream_ptr(stream)))
    return out


def generate_permutation(out, seed: int, base: int = 0, stream=None):
    check(lib.gx_generate_permutation(view(out), seed, base, _stream_ptr(stream)))
    return out
