"""CPU oracle for the operator core — TEST INFRASTRUCTURE ONLY.

Restates the reference engine's operator semantics on the CPU (see the
header of gx_oracle.cpp for the reference file:line each function follows
and how the oracle is pinned).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs may use this package; the product library
never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "gx_oracle.cpp"
LIB = HERE / "liboracle.so"

T_I8, T_I16, T_I32, T_I64, T_B8, T_U8, T_U16, T_U32, T_U64, T_F32, T_F64 = range(1, 12)
NP = {T_I8: np.int8, T_I16: np.int16, T_I32: np.int32, T_I64: np.int64, T_B8: np.bool_, T_U8: np.uint8,
      T_U16: np.uint16, T_U32: np.uint32, T_U64: np.uint64, T_F32: np.float32, T_F64: np.float64}
GX_OF_NP = {np.dtype(v): k for k, v in NP.items()}
SUM, MAX, MIN, AVG, ANY, COUNT_ALL = range(6)


def build() -> Path:
    """Compile gx_oracle.cpp with g++/OpenMP into oracle/liboracle.so."""
    if LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(tmp)]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        vp, i32, i64, f64 = C.c_void_p, C.c_int, C.c_int64, C.c_double
        L.orc_groupby.argtypes = [vp, i32, i64, i32, C.POINTER(vp), C.POINTER(C.c_int), i32, C.POINTER(i64),
                                  C.POINTER(C.c_int), i32, vp, C.POINTER(vp)]
        L.orc_groupby.restype = i64
        L.orc_sort_pairs.argtypes = [vp, i32, i64, vp, i32, i32, i32, i32, i32, vp, vp]
        L.orc_partition_offsets.argtypes = [vp, i32, i64, i32, i32, vp]
        L.orc_join_pairs.argtypes = [vp, i64, vp, i64, i32, vp, vp]
        L.orc_join_pairs.restype = i64
        L.orc_join_count_parallel.argtypes = [vp, i64, vp, i64, i32]
        L.orc_join_count_parallel.restype = i64
        L.orc_join_probe_unique.argtypes = [vp, i64, vp, i64, i32, vp]
        L.orc_join_probe_unique.restype = i64
        L.orc_join_pairs_parallel.argtypes = [vp, i64, vp, i64, i32, vp, vp]
        L.orc_join_pairs_parallel.restype = i64
        L.orc_dict_encode.argtypes = [vp, i32, i64, i32, vp]
        L.orc_dict_encode.restype = i64
        L.orc_dict_with_dict.argtypes = [vp, i64, vp, i64, i32, vp]
        L.orc_ndv_exact.argtypes = [vp, i32, i64]
        L.orc_ndv_exact.restype = i64
        L.orc_hll_registers.argtypes = [vp, i32, i64, i64, vp]
        L.orc_hll_estimate.argtypes = [vp]
        L.orc_hll_estimate.restype = f64
        L.orc_zipf_cdf.argtypes = [i64, f64, vp]
        L.orc_gen_keys.argtypes = [vp, i64, i32, C.c_uint64, C.c_uint64, i32, i32, i64, vp, f64]
        L.orc_gen_values.argtypes = [vp, i64, i32, C.c_uint64, C.c_uint64, i64, i64]
        L.orc_gen_perm.argtypes = [vp, i64, i32, C.c_uint64, i64]
        L.orc_num_threads.restype = i32
        L.orc_set_threads.argtypes = [i32]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def gx_type(a: np.ndarray) -> int:
    return GX_OF_NP[a.dtype]


def out_type(kind: int, t: int) -> int:
    if kind == COUNT_ALL:
        return T_I64
    if kind == AVG:
        return T_F64
    if kind == SUM:
        if t in (T_F32, T_F64):
            return t
        return T_I64 if t in (T_I8, T_I16, T_I32, T_I64) else T_U64
    return t


def groupby(key: np.ndarray, vals: list[np.ndarray], requests: list[tuple[int, int]], agg_count: bool = False):
    """Sorted-by-key group-by: returns [keys, out_0, ..., (+count)]."""
    L = lib()
    key = np.ascontiguousarray(key)
    vals = [np.ascontiguousarray(v) for v in vals]
    n = key.shape[0]
    vt = (C.c_int * max(len(vals), 1))(*[gx_type(v) for v in vals])
    vp = (C.c_void_p * max(len(vals), 1))(*[v.ctypes.data for v in vals])
    rc = (C.c_int64 * max(len(requests), 1))(*[c for c, _ in requests])
    rk = (C.c_int * max(len(requests), 1))(*[k for _, k in requests])
    out_key = np.empty(max(n, 1), dtype=key.dtype)
    outs = []
    for c, k in requests:
        t = T_I64 if k == COUNT_ALL else out_type(k, gx_type(vals[c]))
        outs.append(np.empty(max(n, 1), dtype=NP[t]))
    if agg_count:
        outs.append(np.empty(max(n, 1), dtype=np.int64))
    op = (C.c_void_p * max(len(outs), 1))(*[o.ctypes.data for o in outs])
    g = L.orc_groupby(_p(key), gx_type(key), n, len(vals), vp, vt, len(requests), rc, rk, int(agg_count),
                      _p(out_key), op)
    return [out_key[:g]] + [o[:g] for o in outs]


def sort_pairs(keys: np.ndarray, vals: np.ndarray | None = None, begin_bit=0, end_bit=-1, desc=False,
               iota=False):
    L = lib()
    keys = np.ascontiguousarray(keys)
    n = keys.shape[0]
    ok = np.empty_like(keys)
    ov = None
    if iota:
        ov = np.empty(n, dtype=np.int64)
    elif vals is not None:
        vals = np.ascontiguousarray(vals)
        ov = np.empty_like(vals)
    L.orc_sort_pairs(_p(keys), gx_type(keys), n, _p(vals) if vals is not None else None,
                     vals.dtype.itemsize if vals is not None else 0, int(iota), begin_bit, end_bit, int(desc),
                     _p(ok), _p(ov) if ov is not None else None)
    return ok, ov


def partition_offsets(keys: np.ndarray, b: int, e: int) -> np.ndarray:
    keys = np.ascontiguousarray(keys)
    out = np.empty((1 << (e - b)) + 1, dtype=np.int64)
    lib().orc_partition_offsets(_p(keys), gx_type(keys), keys.shape[0], b, e, _p(out))
    return out


def join_pairs(lkeys: np.ndarray, rkeys: np.ndarray):
    """All (left_row, right_row) with equal keys, sorted."""
    L = lib()
    lkeys, rkeys = np.ascontiguousarray(lkeys), np.ascontiguousarray(rkeys)
    t = gx_type(lkeys)
    m = L.orc_join_pairs(_p(lkeys), lkeys.shape[0], _p(rkeys), rkeys.shape[0], t, None, None)
    ol, orr = np.empty(max(m, 1), np.int64), np.empty(max(m, 1), np.int64)
    L.orc_join_pairs(_p(lkeys), lkeys.shape[0], _p(rkeys), rkeys.shape[0], t, _p(ol), _p(orr))
    return ol[:m], orr[:m]


def join_probe_unique(lkeys: np.ndarray, rkeys: np.ndarray) -> np.ndarray:
    """For a left side with unique keys: match[j] = left row equal to right
    row j, or -1.  The join's pairs are (match[j], j) where match[j] >= 0."""
    lkeys, rkeys = np.ascontiguousarray(lkeys), np.ascontiguousarray(rkeys)
    match = np.empty(rkeys.shape[0], dtype=np.int64)
    rc = lib().orc_join_probe_unique(_p(lkeys), lkeys.shape[0], _p(rkeys), rkeys.shape[0], gx_type(lkeys),
                                     _p(match))
    if rc != 0:
        raise ValueError("join_probe_unique: left keys are not unique")
    return match


def join_pairs_parallel(lkeys: np.ndarray, rkeys: np.ndarray):
    """All (left_row, right_row) pairs with equal keys in right-row order
    (the parallel CPU join baseline; sort them for the canonical order)."""
    L = lib()
    lkeys, rkeys = np.ascontiguousarray(lkeys), np.ascontiguousarray(rkeys)
    t = gx_type(lkeys)
    m = L.orc_join_pairs_parallel(_p(lkeys), lkeys.shape[0], _p(rkeys), rkeys.shape[0], t, None, None)
    ol, orr = np.empty(max(m, 1), np.int64), np.empty(max(m, 1), np.int64)
    L.orc_join_pairs_parallel(_p(lkeys), lkeys.shape[0], _p(rkeys), rkeys.shape[0], t, _p(ol), _p(orr))
    return ol[:m], orr[:m]


def join_count_parallel(lkeys: np.ndarray, rkeys: np.ndarray) -> int:
    return int(lib().orc_join_count_parallel(_p(lkeys), lkeys.shape[0], _p(rkeys), rkeys.shape[0], gx_type(lkeys)))


def dict_encode(keys: np.ndarray, ordered: bool = False):
    keys = np.ascontiguousarray(keys)
    codes = np.empty(keys.shape[0], dtype=np.int64)
    nd = lib().orc_dict_encode(_p(keys), gx_type(keys), keys.shape[0], int(ordered), _p(codes))
    return codes, int(nd)


def dict_with_dict(keys: np.ndarray, dictionary: np.ndarray) -> np.ndarray:
    keys, dictionary = np.ascontiguousarray(keys), np.ascontiguousarray(dictionary)
    out = np.empty(keys.shape[0], dtype=np.int32)
    lib().orc_dict_with_dict(_p(keys), keys.shape[0], _p(dictionary), dictionary.shape[0], gx_type(keys), _p(out))
    return out


def ndv_exact(keys: np.ndarray) -> int:
    keys = np.ascontiguousarray(keys)
    return int(lib().orc_ndv_exact(_p(keys), gx_type(keys), keys.shape[0]))


def hll_registers(keys: np.ndarray, n: int | None = None, stride: int = 1) -> np.ndarray:
    keys = np.ascontiguousarray(keys)
    regs = np.zeros(1 << 13, dtype=np.uint32)
    n = keys.shape[0] if n is None else n
    lib().orc_hll_registers(_p(keys), gx_type(keys), n, stride, _p(regs))
    return regs


def hll_estimate(regs: np.ndarray) -> float:
    return float(lib().orc_hll_estimate(_p(np.ascontiguousarray(regs, dtype=np.uint32))))


def zipf_cdf(groups: int, s: float) -> np.ndarray:
    out = np.empty(groups, dtype=np.float64)
    lib().orc_zipf_cdf(groups, s, _p(out))
    return out


DIST_UNIFORM, DIST_CYCLIC, DIST_ZIPF, DIST_SEQUENCE = range(4)


def gen_keys(n: int, dtype, seed=42, stream_id=0, dist=DIST_UNIFORM, scatter=0, groups=1, zipf_s=0.0,
             miss_frac=0.0, cdf: np.ndarray | None = None) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    if dist == DIST_ZIPF and cdf is None:
        cdf = zipf_cdf(groups, zipf_s)
    lib().orc_gen_keys(_p(out), n, out.dtype.itemsize, seed, stream_id, dist, scatter, groups,
                       _p(cdf) if cdf is not None else None, miss_frac)
    return out


def gen_values(n: int, dtype, seed=42, stream_id=1, lo=0, hi=1) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    lib().orc_gen_values(_p(out), n, gx_type(out), seed, stream_id, lo, hi)
    return out


def gen_perm(n: int, dtype, seed: int, base: int = 0) -> np.ndarray:
    out = np.empty(n, dtype=dtype)
    lib().orc_gen_perm(_p(out), n, out.dtype.itemsize, seed, base)
    return out


def num_threads() -> int:
    return int(lib().orc_num_threads())
