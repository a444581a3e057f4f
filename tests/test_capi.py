"""C ABI checks that need no GPU: the library loads, exports every entry
point include/gx.h declares, and the Python ctypes mirrors of the C structs
have the C layout (checked against a tiny program compiled with gcc)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

import eiger_b200 as gx

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gx.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(gx_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_reference_surface():
    names = declared_functions()
    for must in ("gx_groupby", "gx_groupby_hash", "gx_groupby_sort", "gx_groupby_sort_gfur", "gx_groupby_partition",
                 "gx_groupby_partition_gfur", "gx_inner_eq_join", "gx_sort_column_pair", "gx_sort_column",
                 "gx_argsort", "gx_partition_column_pair", "gx_partition_column", "gx_arg_partition",
                 "gx_compute_partition_offsets", "gx_dictionary_encode", "gx_dictionary_encode_with_order",
                 "gx_dictionary_encode_with_dict", "gx_compute_ndv_approx", "gx_table_free", "gx_last_error_message"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ROOT / "eiger_b200" / "libgx.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(f'''#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gx_column_view), sizeof(gx_table_view), sizeof(gx_column),
         sizeof(gx_agg_request), sizeof(gx_groupby_hint), sizeof(gx_join_hint), sizeof(gx_gen_spec),
         sizeof(gx_batch_instance), sizeof(gx_batch_result));
  printf("%zu %zu %zu\\n", offsetof(gx_groupby_hint, groupby_algo), offsetof(gx_join_hint, max_out),
         offsetof(gx_gen_spec, zipf_cdf));
  return 0;
}}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    py = [ctypes.sizeof(t) for t in (gx.ColumnView, gx.TableView, gx.OwnedColumn, gx.AggRequest, gx.GroupbyHint,
                                     gx.JoinHint, gx.GenSpec, gx.BatchInstance, gx.BatchResult)]
    assert sizes == py
    assert offs == [gx.GroupbyHint.groupby_algo.offset, gx.JoinHint.max_out.offset, gx.GenSpec.zipf_cdf.offset]


def test_hint_defaults_mirror_reference():
    # groupby_hint defaults (groupby.hpp:27-42): no bound, AUTO, flags off.
    h = gx.make_hint()
    assert h.groups_upper_bound == 2 ** 63 - 1 and h.groupby_algo == gx.AUTO_ALGO
    assert (h.zero_based_ids, h.optimize_sort, h.agg_count, h.enable_skf, h.allow_hash_fallback) == (0, 0, 0, 0, 0)
    j = gx.make_join_hint()
    assert (j.sorted_left, j.unique_left, j.max_out) == (0, 0, 0)


def test_agg_output_types_follow_reference():
    # aggregate.cu:19-53 / agg_func.cuh:20-35.
    f = gx.lib.gx_agg_output_type
    assert f(gx.SUM, gx.INT32) == gx.INT64 and f(gx.SUM, gx.INT8) == gx.INT64
    assert f(gx.SUM, gx.UINT32) == gx.UINT64 and f(gx.SUM, gx.FLOAT32) == gx.FLOAT32
    assert f(gx.MAX, gx.INT16) == gx.INT16 and f(gx.AVG, gx.INT32) == gx.FLOAT64
    assert f(gx.COUNT_ALL, gx.EMPTY) == gx.INT64


def test_errors_are_reported_not_thrown():
    # Invalid arguments come back as a status + message, without a GPU.
    h = gx.make_join_hint(gx.JOIN_AUTO, gx.MAT_GFUR)
    arr = (gx.ColumnView * 2)()
    tv = gx.TableView(arr, 2)
    out = ctypes.c_void_p()
    st = gx.lib.gx_inner_eq_join(ctypes.byref(tv), ctypes.byref(tv), ctypes.byref(h), None, ctypes.byref(out))
    assert st == 1 and "auto selection" in gx.last_error()


def test_cpp_shim_compiles_and_maps_errors_to_exceptions(tmp_path):
    # include/gamax/gamax.hpp restates the reference's C++ operator API
    # (namespace gamax) over the C ABI; a reference caller must compile
    # unchanged and see std::runtime_error for a rejected call, as
    # operators/join/join.cu:33-36 throws for a GFUR hint under AUTO.
    src = tmp_path / "shim.cpp"
    src.write_text('''#include <cstdio>
#include <stdexcept>
#include "gamax/gamax.hpp"
using namespace gamax;
int main() {
  std::vector<column_view> cols{column_view(nullptr, 0, data_type{type_id::INT32}),
                                column_view(nullptr, 0, data_type{type_id::INT32})};
  table_view t(cols);
  join::join_hint h;
  h.mat_algo = join::GFUR;
  try {
    join::inner_eq_join(t, t, h);
  } catch (std::runtime_error const& e) {
    std::printf("caught:%s\\n", e.what());
  }
  groupby::groupby_hint gh;
  std::printf("%d %d %lld\\n", (int)gh.groupby_algo, (int)groupby::agg_output_data_type(
      groupby::aggregation_id::SUM, data_type{type_id::INT32}).id(), (long long)gh.groups_upper_bound);
  return 0;
}
''')
    exe = tmp_path / "shim"
    cuda = Path("/usr/local/cuda/include")
    subprocess.run(["g++", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{cuda}", str(src), "-o", str(exe),
                    f"-L{ROOT / 'eiger_b200'}", "-lgx", f"-Wl,-rpath,{ROOT / 'eiger_b200'}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[0].startswith("caught:") and "auto selection" in out[0]
    algo, sum_type, bound = out[1].split()
    assert int(algo) == 0 and int(sum_type) == int(gx.INT64) and int(bound) == 2 ** 63 - 1


def test_invalid_arguments_are_rejected_with_messages():
    # Host-side validation, the reference's std::runtime_error cases
    # (groupby.cu:68-120, sort.cu, partition.cu, stats_compute.cu): each call
    # returns GX_EINVAL with a message and does no device work.
    cv = gx.ColumnView

    def table(cols):
        arr = (cv * len(cols))(*cols)
        return gx.TableView(arr, len(cols)), arr

    out = ctypes.c_void_p()
    kt, _k = table([cv(None, 10, gx.INT32, 0)])
    short_vt, _v = table([cv(None, 9, gx.INT64, 0)])
    vt, _w = table([cv(None, 10, gx.INT64, 0)])
    req = (gx.AggRequest * 1)(gx.AggRequest(0, gx.SUM))
    bad_req = (gx.AggRequest * 1)(gx.AggRequest(5, gx.SUM))

    def groupby(vals, reqs, algo=gx.HASH):
        h = gx.make_hint(gx.HASH, 10)
        h.groupby_algo = algo
        return gx.lib.gx_groupby(ctypes.byref(kt), ctypes.byref(vals), reqs, 1, ctypes.byref(h), None,
                                 ctypes.byref(out))

    oc, ko, vo = gx.OwnedColumn(), gx.OwnedColumn(), gx.OwnedColumn()
    ndv = ctypes.c_int64()
    cases = [
        (lambda: groupby(short_vt, req), "different row count"),
        (lambda: groupby(vt, req, algo=99), "Unsupported groupby algorithm"),
        (lambda: groupby(vt, bad_req), "out of range"),
        (lambda: gx.lib.gx_compute_partition_offsets(cv(None, 10, gx.INT32, 0), 0, 40, None, ctypes.byref(oc)),
         "bad bit range"),
        (lambda: gx.lib.gx_compute_ndv_approx(cv(None, 10, gx.STRING, 0), None, ctypes.byref(ndv)),
         "unsupported column type"),
        (lambda: gx.lib.gx_sort_column_pair(cv(None, 10, gx.INT32, 0), cv(None, 10, gx.INT64, 0), 0, -1, 7, None, 0,
                                            None, ctypes.byref(ko), ctypes.byref(vo)), "bad order"),
        (lambda: gx.lib.gx_sort_column_pair(cv(None, 10, gx.STRING, 0), cv(None, 10, gx.INT64, 0), 0, -1, 0, None, 0,
                                            None, ctypes.byref(ko), ctypes.byref(vo)), "unsupported key type"),
    ]
    for call, words in cases:
        assert call() == 1, words
        assert words in gx.last_error()


def test_reference_style_caller_compiles_against_all_headers(tmp_path):
    # The C++ caller of the GPU test (groupby, join, sort / partition on
    # gamax::column&, dictionary encode, aggregate, phys::*, pullops::*)
    # compiles and links against the headers and libgx.so without a GPU.
    from tests.test_cpp_caller_gpu import CALLER
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    cuda = Path("/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}", str(src),
                    "-o", str(tmp_path / "caller"), f"-L{ROOT / 'eiger_b200'}", "-lgx", f"-L{cuda / 'lib64'}",
                    "-lcudart"], check=True)
