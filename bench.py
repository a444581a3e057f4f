#!/usr/bin/env python
"""Benchmark of the relational operator core on B200.

Default workload (one "step"): group-by over 2^28 rows (AUTO: variant chosen by
the learned selector with the committed weights; --selector plain for the
reference's NDV rule, --algo to force one) — int32 keys
(scattered, uniform over --groups distinct values), an int64 column uniform
in [0, 2^31) and a float64 column uniform in [0, 1), SUM / COUNT / MIN / MAX
on both value columns (the group-by sweep configuration, one point of it).
Inputs are generated on the device once and stay resident in HBM; they are
5.4 GB, far larger than the 126 MB L2, so no L2 flush is needed between
steps.  The sort-based join of 2^24 unique build keys with 2^28 probe keys
(10% absent) is measured too and reported under "join".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gx|reference]

Prints one JSON line (rank 0).  `--impl reference` times the CPU restatement
of the reference path (the oracle; the reference ships no CPU operators) on
the host cores over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "group-by & join Mrows/s at 2^28 rows, % HBM peak; batched+learned vs plain"


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi samples every 25 ms around the timed region: `ready()`
    waits (bounded) for the first sample so a slow nvidia-smi start cannot
    miss a short region, `window()` marks the region, and the summary keeps
    the samples taken inside it (one interval of slack on each side)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 25

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.INTERVAL_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def ready(self, timeout_s: float = 10.0) -> None:
        end = time.monotonic() + timeout_s
        while self.proc and not self.lines and time.monotonic() < end and self.proc.poll() is None:
            time.sleep(0.01)

    def window(self, t0: float, t1: float) -> None:
        self.t0, self.t1 = t0, t1

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        slack = self.INTERVAL_MS / 1000.0
        picked = [ln for t, ln in self.lines
                  if self.t0 is None or self.t0 - slack <= t <= self.t1 + slack]
        for ln in picked:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# Workload construction (device-side generators)
# ---------------------------------------------------------------------------
def make_groupby_inputs(gx, torch, rows: int, groups: int, seed: int):
    k = torch.empty(rows, dtype=torch.int32, device="cuda")
    gx.generate_keys(k, gx.gen_spec(seed=seed, stream_id=0, groups=groups, scatter=1))
    iv = torch.empty(rows, dtype=torch.int64, device="cuda")
    gx.generate_values(iv, gx.gen_spec(seed=seed, stream_id=1, lo=0, hi=1 << 31))
    fv = torch.empty(rows, dtype=torch.float64, device="cuda")
    gx.generate_values(fv, gx.gen_spec(seed=seed, stream_id=2))
    return k, iv, fv


REQS = None


def groupby_reqs(gx):
    return [(0, gx.SUM), (0, gx.MIN), (0, gx.MAX), (1, gx.SUM), (1, gx.MIN), (1, gx.MAX), (0, gx.COUNT_ALL)]


def time_steps(torch, fn, steps: int, warmup: int, dist=None, marks: list | None = None) -> float:
    """Device time (ms) of `steps` calls, CUDA events on the current stream;
    `marks` (if given) receives the host clock at the start and end of the
    timed steps."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    if marks is not None:
        marks.append(time.monotonic())
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(steps):
        fn()
    b.record(s)
    torch.cuda.synchronize()
    if marks is not None:
        marks.append(time.monotonic())
    ms = a.elapsed_time(b)
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms


def kernel_ms(gx, name: str) -> tuple[float, int]:
    import ctypes
    tot, cnt = ctypes.c_double(), ctypes.c_int64()
    gx.check(gx.lib.gx_profile_read(name.encode(), ctypes.byref(tot), ctypes.byref(cnt)))
    return tot.value, cnt.value


def run_gx(args) -> None:
    import torch
    import eiger_b200 as gx
    import ctypes

    gx.lib.gx_profile_enable.argtypes = [ctypes.c_int32]
    gx.lib.gx_profile_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    gx.lib.gx_profile_reset.argtypes = []

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = dist_mod
    else:
        torch.cuda.set_device(0)
    peaks = measured_peaks()
    rows, G = args.rows, args.groups

    # ----------------------------------------------------------- group-by
    k, iv, fv = make_groupby_inputs(gx, torch, rows, G, seed=42 + rank)
    reqs = groupby_reqs(gx)
    hint_algo = {"auto": gx.AUTO_ALGO, "hash": gx.HASH, "sort": gx.SORT, "partition": gx.PARTITION}[args.algo]
    chosen = {}
    # AUTO with the learned selector (committed weights) unless --selector plain.
    learned = False
    if args.algo == "auto" and args.selector == "learned":
        from eiger_b200 import selector as sel_mod
        learned = sel_mod.install()
    sel = gx.SELECT_LEARNED if learned else gx.SELECT_HEURISTIC

    def step():
        h = gx.make_hint(hint_algo, G, selector=sel)
        t = gx.groupby([k], [iv, fv], reqs, h)
        chosen["algo"], chosen["radix_bits"] = h.groupby_algo, h.radix_bits
        return t

    res = step()
    ngroups = res.num_rows
    step_result = res.numpy_columns()  # checked against the oracle after timing
    del res
    launches0 = gx.kernel_launches()
    gx.lib.gx_profile_reset()
    gx.lib.gx_profile_enable(1)
    with ClockSampler(local) as clk:
        clk.ready()
        marks: list = []
        ms = time_steps(torch, step, args.steps, args.warmup, dist, marks)
        clk.window(marks[0], marks[1])
    gx.lib.gx_profile_enable(0)
    launches = gx.kernel_launches() - launches0
    in_bytes = rows * (4 + 8 + 8)
    out_bytes = ngroups * (4 + 8 * 7)
    # Per-launch algorithmic bytes of each timed kernel: the key and value
    # columns read once (aggregation kernels), read and written once per
    # radix pass (partition scatter).
    kernel_bytes = {"hash_groupby": in_bytes, "partition_aggregate": in_bytes, "segmented_reduce": in_bytes,
                    "partition_scatter": 2 * in_bytes, "radix_scatter": 2 * in_bytes}
    kstats = {name: kernel_ms(gx, name) for name in kernel_bytes}
    gx.lib.gx_profile_reset()
    main_kernel = max(kstats, key=lambda nm: kstats[nm][0])
    prof_steps = args.steps + args.warmup  # profiling covers the warm-up steps too
    kms, kcnt = kstats[main_kernel]
    ms_step = ms / args.steps
    value = world * rows / (ms_step * 1e-3) / 1e6
    k_launch_ms = kms / max(kcnt, 1)
    achieved = kernel_bytes[main_kernel] / (k_launch_ms * 1e-3) / 1e9 if kcnt else None
    algo_name = {gx.HASH: "hash", gx.SORT: "sort", gx.SORT_OPT: "sort_opt", gx.SORT_GFUR: "sort_gfur",
                 gx.PARTITION: "partition", gx.PARTITION_GFUR: "partition_gfur"}.get(chosen.get("algo"), "?")
    # DRAM bytes per row of the partition plan's two kernels on this workload,
    # from one ncu capture at 2^25 rows (dram__bytes_read.sum + dram__bytes_write.sum
    # per launch ÷ 2^25; DRAM bytes grow in proportion to rows), scaled to this run:
    #   ncu --set full --clock-control none -k regex:k_units_dense -s 2 -c 1 python bench.py \
    #       --rows 33554432 --steps 2 --warmup 3 --no-join --batch-instances 0 --no-cpu --no-check --no-sweep
    #   ncu --set full --clock-control none -k regex:k_part_scatter_bulk -s 2 -c 1 python bench.py \
    #       --rows 33554432 --steps 3 --warmup 3 --no-join --batch-instances 0 --no-cpu
    # k_units_dense 677.53 + 7.17 MB, k_part_scatter_bulk 688.36 + 621.05 MB (the scatter's
    # last writes leave L2 after the kernel ends).
    dram_per_row = {"partition_aggregate": (677.53e6 + 7.17e6) / 2**25,
                    "partition_scatter": (688.36e6 + 621.05e6) / 2**25}
    traffic = args.traffic
    if traffic is None and main_kernel in dram_per_row and G == 1 << 16 and algo_name.startswith("partition"):
        traffic = dram_per_row[main_kernel] * rows
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"] if achieved else None, "traffic": traffic,
                "kernel": main_kernel, "kernel_ms": k_launch_ms, "launches_per_step": kcnt / prof_steps,
                "kernel_share_of_step": kms / prof_steps / max(ms_step, 1e-9), "peak_source": peaks["source"],
                "kernels_ms_per_step": {nm: round(t / prof_steps, 4) for nm, (t, c) in kstats.items() if c},
                "operator_frac": (in_bytes + out_bytes) / (ms_step * 1e-3) / 1e9 / peaks["hbm_gbs"]}

    # ------------------------------------------------------------- e2e
    hk = torch.empty(rows, dtype=torch.int32, pin_memory=True)
    hiv = torch.empty(rows, dtype=torch.int64, pin_memory=True)
    hfv = torch.empty(rows, dtype=torch.float64, pin_memory=True)
    hk.copy_(k)
    hiv.copy_(iv)
    hfv.copy_(fv)
    del k, iv, fv
    torch.cuda.empty_cache()

    def e2e_step():
        dk = hk.to("cuda", non_blocking=True)
        div = hiv.to("cuda", non_blocking=True)
        dfv = hfv.to("cuda", non_blocking=True)
        t = gx.groupby([dk], [div, dfv], reqs, gx.make_hint(hint_algo, G, selector=sel))
        cols = t.numpy_columns()  # device -> host read of the result
        return cols

    e2e_steps = max(1, min(args.steps, 3))
    e2e_ms = time_steps(torch, e2e_step, e2e_steps, 1, dist) / e2e_steps
    e2e = {"value": world * rows / (e2e_ms * 1e-3) / 1e6, "unit": "Mrows/s", "h2d_bytes_per_step": in_bytes,
           "d2h_bytes_per_step": out_bytes, "ms_per_step": e2e_ms}
    # ------------------------------------------- oracle check + CPU baseline
    # The oracle (CPU restatement, all host threads) on the same host copies
    # of the timed workload: it checks the step's output column by column and
    # its time is the CPU baseline on the full workload.
    parity, cpu = None, None
    if rank == 0 and not args.no_check:
        parity, cpu = check_against_oracle(step_result, hk.numpy(), hiv.numpy(), hfv.numpy())
        if world > 1:
            cpu = None  # CPU baseline on single-GPU runs only
    del hk, hiv, hfv
    torch.cuda.empty_cache()

    # ------------------------------------------------------------- join
    join = None
    if not args.no_join:
        nb, npr = 1 << 24, args.join_rows
        bk = torch.empty(nb, dtype=torch.int32, device="cuda")
        gx.generate_permutation(bk, 42 + rank)
        brow = torch.arange(nb, dtype=torch.int64, device="cuda")
        pk = torch.empty(npr, dtype=torch.int32, device="cuda")
        gx.generate_keys(pk, gx.gen_spec(seed=39 + rank, groups=nb, miss_frac=0.1))
        prow = torch.arange(npr, dtype=torch.int64, device="cuda")
        jh = gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, unique_left=1)
        nsteps = max(1, args.steps // 2)

        def measure(fn, alg_bytes_of):
            r = fn()
            matches = r.num_rows
            del r
            gx.lib.gx_profile_reset()
            gx.lib.gx_profile_enable(1)
            ms = time_steps(torch, fn, nsteps, 3, dist) / nsteps
            gx.lib.gx_profile_enable(0)
            wms, wc = kernel_ms(gx, "join_probe_write")
            cms, cc = kernel_ms(gx, "join_probe_count")
            gx.lib.gx_profile_reset()
            alg = alg_bytes_of(matches)
            probe_ms = wms / max(wc, 1) + cms / max(cc, 1)
            return {"value": world * (nb + npr) / (ms * 1e-3) / 1e6, "unit": "Mrows/s", "ms_per_step": ms,
                    "matches": matches, "probe_write_ms": wms / max(wc, 1), "probe_count_ms": cms / max(cc, 1),
                    "probe_frac": alg / (probe_ms * 1e-3) / 1e9 / peaks["hbm_gbs"] if wc else None,
                    "operator_frac": alg / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"],
                    "algorithmic_bytes": alg}

        # Row-id pairs (build_rowid, probe_rowid): |R|*4 + |S|*4 + M*16 bytes.
        join = measure(lambda: gx.inner_eq_join_rowids(bk, pk, jh), lambda m: (nb + npr) * 4 + m * 16)
        join["workload"] = (f"sort-based inner equi-join, 2^24 unique int32 build keys x {npr} int32 probe keys "
                            "(10% absent); output (build_rowid, probe_rowid) int64 pairs")
        # Table form [key, build payload, probe payload] with int64 payloads.
        join["table_form"] = measure(lambda: gx.inner_eq_join([bk, brow], [pk, prow], jh),
                                     lambda m: (nb + npr) * 12 + m * 20)
        # Second probe set: Zipf s = 1.0 over the build keys (rank r -> the
        # r-th build key, so hot probe keys are spread over the key space).
        cdf = torch.from_numpy(gx.zipf_cdf(nb, 1.0)).cuda()
        zr = torch.empty(npr, dtype=torch.int32, device="cuda")
        gx.generate_keys(zr, gx.gen_spec(seed=41 + rank, dist=gx.DIST_ZIPF, groups=nb, zipf_s=1.0,
                                         zipf_cdf=cdf.data_ptr()))
        zpk = bk[zr.long()]
        del zr, cdf
        join["zipf_1.0"] = measure(lambda: gx.inner_eq_join_rowids(bk, zpk, jh), lambda m: (nb + npr) * 4 + m * 16)
        del zpk
        # The hash multiset (join_algo HASH) and the partitioned hash join
        # (join_algo PARTITION) on the same keys.
        for algo, nm in ((gx.JOIN_HASH, "hash"), (gx.JOIN_PARTITION, "partition_hash")):
            h3 = gx.make_join_hint(algo, gx.MAT_GFUR, unique_left=1)
            join[nm] = measure(lambda: gx.inner_eq_join_rowids(bk, pk, h3), lambda m: (nb + npr) * 4 + m * 16)
        # The sorted-build matcher: the same join with keys spread 8 apart, so
        # the build side is too sparse for direct placement; sorted build run
        # + radix directory (SORTED_BUILD) and both sides sorted (SORT_MERGE).
        sbk, spk = bk * 8, pk * 8
        for mode, nm in ((gx.SORTED_BUILD, "sorted_build"), (gx.SORT_MERGE, "sort_merge")):
            h2 = gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, unique_left=1, sort_mode=mode)
            join[nm] = measure(lambda: gx.inner_eq_join_rowids(sbk, spk, h2), lambda m: (nb + npr) * 4 + m * 16)
        del sbk, spk
        if rank == 0 and world == 1 and not args.no_cpu:
            join["cpu_baseline"] = cpu_join_baseline(bk.cpu().numpy(), pk.cpu().numpy())
        del bk, brow, pk, prow

    # ------------------------------------------------------- sweep grid
    # The group-by sweep at the timed row count, every variant: G over the
    # sweep's range (int32 keys, uniform), plus Zipf 1.5 and int64 keys.
    sweep = shapes = operators = None
    if not args.no_sweep:
        sweep = sweep_grid(gx, torch, rows, peaks, dist)
        shapes = shapes_grid(gx, torch, rows, peaks, sel, dist)
        operators = operators_grid(gx, torch, rows, peaks, dist)

    # ----------------------------------------------------------- batched
    batched = None
    if args.batch_instances > 0:
        from eiger_b200 import batch as B
        insts, _ = B.make_instances(args.batch_instances, seed=11 + rank)
        total = sum(it.rows for it in insts)
        plan = B.Plan(insts, max_distinct=10_000)
        tile, lf = plan.tuning()
        nsteps = max(1, args.steps // 2)
        l0 = gx.kernel_launches()
        b_ms = time_steps(torch, plan.run, nsteps, 3, dist) / nsteps
        b_launches = (gx.kernel_launches() - l0) // (nsteps + 3)
        l0 = gx.kernel_launches()
        p_ms = time_steps(torch, plan.run_per_instance, nsteps, 3, dist) / nsteps
        p_launches = (gx.kernel_launches() - l0) // (nsteps + 3)
        # Input bytes: every instance's strings, offsets, dates and amounts
        # once (what the per-instance engine reads).  Must-read bytes of a
        # plan that applies the date range first: dates and offsets of every
        # row, strings and amounts of the kept rows only.
        in_b = sum(int(it.offsets[-1].item()) + (it.rows + 1) * 8 + it.rows * 12 for it in insts)
        need_b = 0
        for it in insts:
            keep = (it.date >= it.lo) & (it.date < it.hi)
            lens = it.offsets[1:] - it.offsets[:-1]
            need_b += (it.rows + 1) * 8 + it.rows * 4 + int((lens * keep).sum().item()) + 8 * int(keep.sum().item())
        batched = {
            "workload": (f"{len(insts)} string group-by pipelines, rows log-uniform in [2^12, 2^22] "
                         f"({total} rows total): dictionary-encode ASCII keys (10^4 distinct, 8..32 bytes), "
                         "keep 40% of rows by a date range, SUM(int64 scale-2 decimal) + COUNT per key"),
            "rows": total, "input_bytes": in_b, "must_read_bytes": need_b,
            "batched": {"ms_per_step": b_ms, "value": world * total / (b_ms * 1e-3) / 1e6, "unit": "Mrows/s",
                        "launches_per_step": b_launches, "hbm_frac": in_b / (b_ms * 1e-3) / 1e9 / peaks["hbm_gbs"],
                        "hbm_frac_must_read": need_b / (b_ms * 1e-3) / 1e9 / peaks["hbm_gbs"]},
            "per_instance": {"ms_per_step": p_ms, "value": world * total / (p_ms * 1e-3) / 1e6, "unit": "Mrows/s",
                             "launches_per_step": p_launches},
            "speedup": p_ms / b_ms, "tile_rows": tile, "load_factor_pct": lf,
        }
        del plan, insts
        torch.cuda.empty_cache()

    # ------------------------------------------------------ cpu baseline
    if cpu is None and rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_groupby_baseline(args.cpu_rows, G)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mrows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "config": {"workload": f"group-by ({args.algo}: ran {algo_name}), {rows} rows, int32 keys uniform over "
                                   f"{G} scattered values, int64 [0,2^31) + float64 [0,1) values, "
                                   "SUM/COUNT/MIN/MAX on both",
                       "rows": rows, "groups": G, "groups_found": ngroups, "algo": args.algo,
                       "variant_run": algo_name, "radix_bits": chosen.get("radix_bits"),
                       "selector": "learned" if learned else ("plain" if args.algo == "auto" else "forced"),
                       "l2": "inputs (5.4 GB) larger than L2; no flush"},
            "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary(), "join": join, "batched": batched, "sweep": sweep, "shapes": shapes,
            "operators": operators,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def sweep_grid(gx, torch, rows: int, peaks: dict, dist=None) -> list:
    """HASH / SORT / PARTITION over a grid of group counts and skews, 7
    aggregates, at `rows` rows: ms, Grows/s and fraction of measured HBM per
    point (algorithmic bytes rows * (K + 16) + groups * (K + 56))."""
    reqs = groupby_reqs(gx)
    points = [("int32", 0.0, 1 << g) for g in (4, 10, 16, 20, 24, 26)]
    points += [("int32", 1.5, 1 << 20), ("int64", 0.0, 1 << 16), ("int64", 1.5, 1 << 24)]
    out = []
    for kdt, z, G in points:
        k = torch.empty(rows, dtype=torch.int32 if kdt == "int32" else torch.int64, device="cuda")
        cdf = None
        if z > 0:
            cdf = torch.from_numpy(gx.zipf_cdf(G, z)).cuda()
            spec = gx.gen_spec(seed=1, dist=gx.DIST_ZIPF, groups=G, zipf_s=z, scatter=1, zipf_cdf=cdf.data_ptr())
        else:
            spec = gx.gen_spec(seed=1, groups=G, scatter=1)
        gx.generate_keys(k, spec)
        iv = torch.empty(rows, dtype=torch.int64, device="cuda")
        gx.generate_values(iv, gx.gen_spec(seed=1, stream_id=1, lo=0, hi=1 << 31))
        fv = torch.empty(rows, dtype=torch.float64, device="cuda")
        gx.generate_values(fv, gx.gen_spec(seed=1, stream_id=2))
        kb = 4 if kdt == "int32" else 8
        for name, algo in (("hash", gx.HASH), ("sort", gx.SORT), ("partition", gx.PARTITION)):
            def step():
                return gx.groupby([k], [iv, fv], reqs, gx.make_hint(algo, G))
            r = step()
            ng = r.num_rows
            del r
            ms = time_steps(torch, step, 2, 1, dist) / 2
            alg = rows * (kb + 16) + ng * (kb + 56)
            out.append({"key": kdt, "zipf": z, "groups": G, "algo": name, "ms": round(ms, 3),
                        "grows_s": round(rows / ms / 1e6, 2),
                        "hbm_frac": round(alg / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4)})
        del k, iv, fv, cdf
        torch.cuda.empty_cache()
    return out


def shapes_grid(gx, torch, rows: int, peaks: dict, sel: int, dist=None) -> list:
    """Group-by requests outside the compiled aggregation plans, through
    AUTO at `rows` rows: a run-time aggregation list over the int64 + float64
    columns (2^16 and 2^10 groups), and three value columns (int64, float64,
    int32: four moved columns, 24 B per row, in the partition scatter).  Per
    shape: AUTO's pick with its ms, Grows/s and
    fraction of measured HBM (algorithmic bytes: every input column read
    once plus the output records), and the ms of HASH and PARTITION forced."""
    names = {gx.HASH: "hash", gx.SORT: "sort", gx.SORT_OPT: "sort_opt", gx.SORT_GFUR: "sort_gfur",
             gx.PARTITION: "partition", gx.PARTITION_GFUR: "partition_gfur"}
    iv = torch.empty(rows, dtype=torch.int64, device="cuda")
    gx.generate_values(iv, gx.gen_spec(seed=5, stream_id=1, lo=0, hi=1 << 31))
    fv = torch.empty(rows, dtype=torch.float64, device="cuda")
    gx.generate_values(fv, gx.gen_spec(seed=5, stream_id=2))
    i32 = torch.empty(rows, dtype=torch.int32, device="cuda")
    gx.generate_values(i32, gx.gen_spec(seed=5, stream_id=3, lo=-(1 << 20), hi=1 << 20))
    generic = [(1, gx.SUM), (0, gx.MAX), (0, gx.COUNT_ALL)]
    three = [(0, gx.SUM), (1, gx.SUM), (2, gx.MIN), (2, gx.MAX), (0, gx.COUNT_ALL)]
    shapes = [("sum f64, max i64, count", 1 << 16, [iv, fv], generic, 2),
              ("sum f64, max i64, count", 1 << 10, [iv, fv], generic, 2),
              ("sum i64, sum f64, min/max i32, count (3 value columns)", 1 << 16, [iv, fv, i32], three, 4)]
    out = []
    for desc, G, cols, reqs, n_out in shapes:
        k = torch.empty(rows, dtype=torch.int32, device="cuda")
        gx.generate_keys(k, gx.gen_spec(seed=5, groups=G, scatter=1))
        chosen = {}

        def step():
            h = gx.make_hint(gx.AUTO_ALGO, G, selector=sel)
            t = gx.groupby([k], cols, reqs, h)
            chosen["algo"] = h.groupby_algo
            return t

        r = step()
        ng = r.num_rows
        del r
        ms = time_steps(torch, step, 3, 2, dist) / 3
        alg = rows * (4 + sum(c.element_size() for c in cols)) + ng * (4 + 8 * n_out)
        forced = {}
        for name, algo in (("hash", gx.HASH), ("partition", gx.PARTITION)):
            forced[name + "_ms"] = round(time_steps(
                torch, lambda: gx.groupby([k], cols, reqs, gx.make_hint(algo, G)), 3, 2, dist) / 3, 3)
        out.append({"aggregates": desc, "groups": G, "groups_found": ng, "algo": names.get(chosen["algo"], "?"),
                    "ms": round(ms, 3), "grows_s": round(rows / ms / 1e6, 2),
                    "hbm_frac": round(alg / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4), **forced})
        del k
    del iv, fv, i32
    torch.cuda.empty_cache()
    return out


def operators_grid(gx, torch, rows: int, peaks: dict, dist=None) -> list:
    """The operators beside the group-by, each on its own at `rows` rows
    (int32 keys uniform over 2^16 scattered values, int64 values in
    [0, 2^31)): radix sort and 8-bit radix partition of (key, value) pairs,
    dictionary encode, the HyperLogLog distinct estimate, and a BETWEEN
    filter keeping half the rows with the compaction of both columns.  Per
    operator (its C-ABI call): ms, Grows/s and the fraction of measured HBM
    for its algorithmic bytes (inputs read once, outputs written once; a
    4-pass sort moves about four times that)."""
    k = torch.empty(rows, dtype=torch.int32, device="cuda")
    gx.generate_keys(k, gx.gen_spec(seed=11, groups=1 << 16, scatter=1))
    v = torch.empty(rows, dtype=torch.int64, device="cuda")
    gx.generate_values(v, gx.gen_spec(seed=11, stream_id=1, lo=0, hi=1 << 31))
    pair = rows * (4 + 8)
    half = [gx.predicate(1, gx.CMP_BETWEEN, 0, 1 << 30)]
    import ctypes
    kv, vv = gx.view(k), gx.view(v)

    # Each operator through its C-ABI call, as a C caller sees it: outputs
    # stay in the library's buffers and are freed after the call (the Python
    # wrappers' copies into torch tensors are not the operator).
    def c_pair(fn, *args):
        ko, vo = gx.OwnedColumn(), gx.OwnedColumn()
        gx.check(fn(kv, vv, *args, None, 0, None, ctypes.byref(ko), ctypes.byref(vo)))
        gx.check(gx.lib.gx_free(ko.data, None))
        gx.check(gx.lib.gx_free(vo.data, None))

    def c_dict():
        o, nd = gx.OwnedColumn(), ctypes.c_int64()
        gx.check(gx.lib.gx_dictionary_encode(kv, gx.INT32, 0, 0.25, None, ctypes.byref(o), ctypes.byref(nd)))
        gx.check(gx.lib.gx_free(o.data, None))

    ops = [("radix sort, 32 key bits (int32 key, int64 value)",
            lambda: c_pair(gx.lib.gx_sort_column_pair, 0, -1, gx.ASCENDING), 2 * pair),
           ("radix partition, 8 bits (int32 key, int64 value)",
            lambda: c_pair(gx.lib.gx_partition_column_pair, 0, 8), 2 * pair),
           ("dictionary encode (int32 keys -> int32 codes)", c_dict, rows * 8),
           ("HyperLogLog distinct estimate (int32 keys)", lambda: gx.compute_ndv_approx(k), rows * 4),
           ("filter: int64 BETWEEN keeping 1/2, compaction of both columns", lambda: gx.select([k, v], half),
            pair + pair // 2)]
    out = []
    for desc, fn, alg in ops:
        ms = time_steps(torch, fn, 3, 2, dist) / 3
        out.append({"op": desc, "ms": round(ms, 3), "grows_s": round(rows / ms / 1e6, 2),
                    "hbm_frac": round(alg / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4)})
    del k, v
    torch.cuda.empty_cache()
    return out


def run_sweep(args) -> None:
    """Group-by sweep (rows fixed, distinct count and skew swept) over the
    HASH / SORT / PARTITION variants; one JSON line per point."""
    import torch
    import eiger_b200 as gx

    torch.cuda.set_device(0)
    peaks = measured_peaks()
    rows = args.rows
    gs = [int(g) for g in args.sweep_groups.split(",")]
    zs = [float(z) for z in args.sweep_zipf.split(",")]
    algos = {"hash": gx.HASH, "sort": gx.SORT, "partition": gx.PARTITION}
    reqs = groupby_reqs(gx)
    if args.sweep_reqs == "sumcount":
        reqs = [(0, gx.SUM), (0, gx.COUNT_ALL)]
    for kdt in args.sweep_keys.split(","):
        tdt = torch.int32 if kdt == "int32" else torch.int64
        for z in zs:
            for G in gs:
                k = torch.empty(rows, dtype=tdt, device="cuda")
                cdf = None
                if z > 0:
                    cdf = torch.from_numpy(gx.zipf_cdf(G, z)).cuda()
                    spec = gx.gen_spec(seed=1, dist=gx.DIST_ZIPF, groups=G, zipf_s=z, scatter=1,
                                       zipf_cdf=cdf.data_ptr())
                else:
                    spec = gx.gen_spec(seed=1, groups=G, scatter=1)
                gx.generate_keys(k, spec)
                iv = torch.empty(rows, dtype=torch.int64, device="cuda")
                gx.generate_values(iv, gx.gen_spec(seed=1, stream_id=1, lo=0, hi=1 << 31))
                fv = torch.empty(rows, dtype=torch.float64, device="cuda")
                gx.generate_values(fv, gx.gen_spec(seed=1, stream_id=2))
                kb = 4 if kdt == "int32" else 8
                for name in args.sweep_algos.split(","):
                    algo = algos[name]

                    def step():
                        return gx.groupby([k], [iv, fv], reqs, gx.make_hint(algo, G))
                    try:
                        r = step()
                        ng = r.num_rows
                        del r
                        ms = time_steps(torch, step, args.steps, 2) / args.steps
                        vb, ob = (8, 16) if args.sweep_reqs == "sumcount" else (16, 56)
                        alg = rows * (kb + vb) + ng * (kb + ob)
                        print(json.dumps({"key": kdt, "zipf": z, "groups": G, "algo": name, "ms": round(ms, 3),
                                          "mrows_s": round(rows / ms / 1e3, 1),
                                          "hbm_frac": round(alg / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"], 4),
                                          "groups_found": ng}), flush=True)
                    except Exception as e:  # report and continue the sweep
                        print(json.dumps({"key": kdt, "zipf": z, "groups": G, "algo": name, "error": str(e)}),
                              flush=True)
                del k, iv, fv, cdf
                torch.cuda.empty_cache()


def run_join_only(args) -> None:
    """The C3 rowid join alone (for profiling captures): 2^24 unique build
    keys x --join-rows probe keys (10% absent); prints one JSON line."""
    import torch
    import eiger_b200 as gx
    torch.cuda.set_device(0)
    nb, npr = 1 << 24, args.join_rows
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    gx.generate_permutation(bk, 42)
    pk = torch.empty(npr, dtype=torch.int32, device="cuda")
    gx.generate_keys(pk, gx.gen_spec(seed=39, groups=nb, miss_frac=0.1))
    mode = args.join_mode
    if mode in ("sorted_build", "sort_merge"):
        # keys spread 8 apart: too sparse for direct placement
        bk, pk = bk * 8, pk * 8
        jh = gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, unique_left=1,
                               sort_mode=gx.SORTED_BUILD if mode == "sorted_build" else gx.SORT_MERGE)
    elif mode in ("hash", "partition_hash"):
        jh = gx.make_join_hint(gx.JOIN_HASH if mode == "hash" else gx.JOIN_PARTITION, gx.MAT_GFUR, unique_left=1)
    else:
        jh = gx.make_join_hint(gx.JOIN_SORT, gx.MAT_GFUR, unique_left=1)
    ms = time_steps(torch, lambda: gx.inner_eq_join_rowids(bk, pk, jh), args.steps, args.warmup) / args.steps
    print(json.dumps({"workload": f"rowid join ({mode}), 2^24 unique int32 build keys x {npr} probe keys "
                      "(10% absent)", "ms_per_step": ms, "value": (nb + npr) / (ms * 1e-3) / 1e6,
                      "unit": "Mrows/s"}), flush=True)


def check_against_oracle(got_cols, k, iv, fv):
    """Compares the timed step's output with the oracle run on the same
    input bytes (keys, counts and integer / MIN / MAX columns bit-exact,
    float64 SUM within 1e-12 relative); the oracle's time on all host threads
    is the CPU baseline on the full workload."""
    import oracle as O
    reqs = [(0, O.SUM), (0, O.MIN), (0, O.MAX), (1, O.SUM), (1, O.MIN), (1, O.MAX), (0, O.COUNT_ALL)]
    t0 = time.perf_counter()
    exp = O.groupby(k, [iv, fv], reqs)
    dt = time.perf_counter() - t0
    order = np.argsort(got_cols[0], kind="stable")
    got = [c[order] for c in got_cols]
    exact, rel = True, 0.0
    for i, (g, e) in enumerate(zip(got, exp)):
        if g.shape != e.shape or g.dtype != e.dtype:
            exact = False
            continue
        if i == 4:  # float64 SUM
            rel = float(np.max(np.abs(g - e) / np.maximum(np.abs(e), 1e-300))) if len(e) else 0.0
        elif not np.array_equal(g, e):
            exact = False
    ok = exact and rel <= 1e-12
    parity = {"ok": ok, "rows": int(k.shape[0]), "groups": int(len(exp[0])), "exact_columns_equal": exact,
              "float64_sum_max_rel_err": rel, "tolerance": 1e-12,
              "check": "step output vs oracle on the same inputs, sorted by key"}
    cpu = {"value": k.shape[0] / dt / 1e6, "unit": "Mrows/s", "cores": O.num_threads(), "kind": "port",
           "sample": f"the full workload ({k.shape[0]} rows): radix-partitioned open-addressing group-by, "
                     "sorted output", "cpu_model": cpu_model()}
    return parity, cpu


def cpu_model() -> str:
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_join_baseline(bk, pk) -> dict:
    """Parallel CPU hash join (oracle) of the rowid join on the same keys."""
    import oracle as O
    t0 = time.perf_counter()
    l, r = O.join_pairs_parallel(bk, pk)
    dt = time.perf_counter() - t0
    return {"value": (len(bk) + len(pk)) / dt / 1e6, "unit": "Mrows/s", "cores": O.num_threads(), "kind": "port",
            "matches": int(len(l)), "sample": "the full join (chained hash build, parallel probe, pairs written)",
            "cpu_model": cpu_model()}


def cpu_groupby_baseline(rows: int, groups: int) -> dict:
    """The oracle (CPU restatement, all host threads) on a bounded sample."""
    import oracle as O
    k = O.gen_keys(rows, np.int32, groups=groups, scatter=1, seed=42)
    iv = O.gen_values(rows, np.int64, seed=42, stream_id=1, lo=0, hi=1 << 31)
    fv = O.gen_values(rows, np.float64, seed=42, stream_id=2)
    reqs = [(0, O.SUM), (0, O.MIN), (0, O.MAX), (1, O.SUM), (1, O.MIN), (1, O.MAX), (0, O.COUNT_ALL)]
    t0 = time.perf_counter()
    O.groupby(k, [iv, fv], reqs)
    dt = time.perf_counter() - t0
    return {"value": rows / dt / 1e6, "unit": "Mrows/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{rows} rows of the same workload (oracle hash group-by, sorted output)"}


def run_reference(args) -> None:
    """CPU restatement of the reference path, host cores, bounded samples."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O
    rows = args.cpu_rows
    G = args.groups
    k = O.gen_keys(rows, np.int32, groups=G, scatter=1, seed=42)
    iv = O.gen_values(rows, np.int64, seed=42, stream_id=1, lo=0, hi=1 << 31)
    fv = O.gen_values(rows, np.float64, seed=42, stream_id=2)
    reqs = [(0, O.SUM), (0, O.MIN), (0, O.MAX), (1, O.SUM), (1, O.MIN), (1, O.MAX), (0, O.COUNT_ALL)]
    for _ in range(args.warmup):
        O.groupby(k, [iv, fv], reqs)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.groupby(k, [iv, fv], reqs)
    dt = (time.perf_counter() - t0) / args.steps
    value = rows / dt / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "config": {"workload": f"group-by (oracle hash aggregation), {args.rows} rows, int32 keys uniform over {G} scattered "
                                   "values, int64 + float64 values, SUM/COUNT/MIN/MAX on both",
                       "rows": args.rows, "groups": G, "sample_rows": rows},
            "cpu_baseline": {"value": value, "unit": "Mrows/s", "cores": O.num_threads(), "kind": "port",
                             "sample": f"{rows} rows per step (the reference has no CPU operators; this is "
                                       "the CPU restatement of its group-by)", "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": "Mrows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gx", "reference"], default="gx")
    ap.add_argument("--rows", type=int, default=1 << 28)
    ap.add_argument("--groups", type=int, default=1 << 16)
    ap.add_argument("--algo", choices=["auto", "hash", "sort", "partition"], default="auto",
                    help="group-by variant (auto: the engine's plain selection rule)")
    ap.add_argument("--join-rows", type=int, default=1 << 28)
    ap.add_argument("--no-join", action="store_true")
    ap.add_argument("--join-only", action="store_true", help="only the rowid join (profiling captures)")
    ap.add_argument("--join-mode", default="auto", choices=["auto", "sorted_build", "sort_merge", "hash",
                                                             "partition_hash"],
                    help="matcher of --join-only: auto (dense placement when the build keys allow it), the "
                         "sorted-build or sort-merge matcher on keys spread 8 apart, or the hash joins")
    ap.add_argument("--selector", choices=["learned", "plain"], default="learned",
                    help="AUTO's chooser: the learned FP16 MLP (committed weights) or the plain NDV rule")
    ap.add_argument("--batch-instances", type=int, default=512, help="batched pipeline instances (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true", help="skip the oracle check of the timed step's output")
    ap.add_argument("--no-sweep", action="store_true", help="skip the group-by sweep grid in the bench line")
    ap.add_argument("--cpu-rows", type=int, default=1 << 24)
    ap.add_argument("--traffic", type=float, default=None,
                    help="dram bytes per launch of the dominant kernel from an ncu capture")
    ap.add_argument("--sweep", action="store_true", help="group-by sweep over variants, groups and skew")
    ap.add_argument("--sweep-groups", default=",".join(str(1 << b) for b in range(4, 27, 2)))
    ap.add_argument("--sweep-zipf", default="0")
    ap.add_argument("--sweep-keys", default="int32")
    ap.add_argument("--sweep-algos", default="hash,sort,partition")
    ap.add_argument("--sweep-reqs", default="all", choices=["all", "sumcount"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.sweep:
        run_sweep(args)
        return
    if args.join_only:
        run_join_only(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gx(args)


if __name__ == "__main__":
    main()
