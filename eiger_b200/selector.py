"""Learned group-by strategy selector: data collection, training, loading.

The selector scores the HASH / SORT / PARTITION group-by variants (and four
partition fan-outs) from a sketch of a 2^14-row key sample
(gx_selector_features).  Its network is a 3-layer FP16 MLP trained on the
GPU with the library's own kernels (gx_mlp_forward_backward and
gx_mlp_adam_step) on timings the plain engine produces for synthetic
instances.  The plain NDV rule of the reference (HLL estimate <= 2^14 for
4-byte keys / 2^18 for 8-byte keys -> HASH, else PARTITION) stays the
fallback and the baseline for regret.

    python -m eiger_b200.selector collect --instances 4096 --out timings.npz
    python -m eiger_b200.selector train timings.npz --out eiger_b200/selector_weights.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time
from pathlib import Path

import numpy as np

F, H, O = 20, 64, 7
KF = 16              # key-sample features; the last 4 describe the aggregation list
NV = 3               # variants: HASH, SORT, PARTITION
FANOUTS = [8, 10, 12, 14]
WEIGHTS = Path(__file__).resolve().parent / "selector_weights.npz"


def _gx():
    import eiger_b200 as gx
    return gx


def param_count() -> int:
    return int(_gx().lib.gx_selector_param_count())


# ---------------------------------------------------------------------------
# Instances (C4: rows log-uniform in 2^16..2^28, NDV log-uniform in 1..rows,
# Zipf s uniform in [0, 2], int32 or int64 keys).  Half the instances run
# SUM + COUNT of an int64 column, half SUM / MIN / MAX of an int64 and a
# float64 column plus COUNT (the benchmark's aggregation list).
# ---------------------------------------------------------------------------
AGGS = {"sumcount": [(0, 0), (0, 5)],
        "seven": [(0, 0), (0, 2), (0, 1), (1, 0), (1, 2), (1, 1), (0, 5)]}  # (column, gx agg kind)
def draw_instances(count: int, seed: int, min_log2=16, max_log2=28) -> list[dict]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        rows = int(2 ** rng.uniform(min_log2, max_log2))
        ndv = int(max(1, round(2 ** rng.uniform(0, math.log2(rows)))))
        out.append({"rows": rows, "ndv": ndv, "zipf": float(rng.uniform(0, 2)),
                    "key": "int64" if rng.random() < 0.5 else "int32", "seed": int(seed * 100003 + i),
                    "aggs": "seven" if rng.random() < 0.5 else "sumcount"})
    return out


def make_instance(inst: dict):
    import torch
    gx = _gx()
    rows, G = inst["rows"], inst["ndv"]
    kdt = torch.int32 if inst["key"] == "int32" else torch.int64
    k = torch.empty(rows, dtype=kdt, device="cuda")
    cdf = None
    if inst["zipf"] > 0.01 and G > 1:
        # Closed-form Zipf on the device: a CDF table of up to 2^28 entries
        # would cost seconds per instance to build and to search.
        spec = gx.gen_spec(seed=inst["seed"], dist=gx.DIST_ZIPF_APPROX, groups=G, zipf_s=inst["zipf"], scatter=1)
    else:
        spec = gx.gen_spec(seed=inst["seed"], groups=G, scatter=1)
    gx.generate_keys(k, spec)
    v = torch.empty(rows, dtype=torch.int64, device="cuda")
    gx.generate_values(v, gx.gen_spec(seed=inst["seed"], stream_id=1, lo=0, hi=1 << 31))
    vals = [v]
    if inst.get("aggs", "sumcount") == "seven":
        f = torch.empty(rows, dtype=torch.float64, device="cuda")
        gx.generate_values(f, gx.gen_spec(seed=inst["seed"], stream_id=2))
        vals.append(f)
    return k, vals, cdf


def plan_features(vals, reqs) -> np.ndarray:
    """Features 16..19 (the aggregation list), computed by the library."""
    gx = _gx()
    tv, _keep = gx.table_view(vals)
    arr = (gx.AggRequest * len(reqs))(*[gx.AggRequest(c, k) for c, k in reqs])
    out = np.zeros(F - KF, dtype=np.float32)
    gx.check(gx.lib.gx_selector_plan_features(C.byref(tv), arr, len(reqs), 0, out.ctypes.data))
    return out


def features(key, vals=None, reqs=None) -> np.ndarray:
    gx = _gx()
    f = np.zeros(F, dtype=np.float32)
    gx.check(gx.lib.gx_selector_features(gx.view(key), gx._stream_ptr(None), f.ctypes.data))
    if vals is not None:
        f[KF:] = plan_features(vals, reqs)
    return f


def time_call(fn, reps: int = 1) -> float:
    import torch
    fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / reps * 1e3


def heuristic_algo(key) -> int:
    """The plain AUTO rule (what gx_groupby picks without the selector):
    HASH when the full-column HyperLogLog estimate is at most 2^14 distinct
    keys for 4-byte keys or 2^18 for 8-byte keys, else PARTITION
    (src/cuda/operators/groupby/groupby.cu:68-119)."""
    gx = _gx()
    est = gx.compute_ndv_approx(key)
    thr = (1 << 14) if key.element_size() == 4 else (1 << 18)
    return gx.HASH if est <= thr else gx.PARTITION


def _pack(instances, index, feats, times, ftimes, heur) -> dict:
    return {"index": np.array(index, np.int64),
            "features": np.array(feats, np.float32).reshape(-1, F), "times": np.array(times, np.float64).reshape(-1, NV),
            "fanout_times": np.array(ftimes, np.float64).reshape(-1, len(FANOUTS)),
            "heuristic": np.array(heur, np.int32), "instances": json.dumps([instances[i] for i in index])}


def collect(instances: list[dict], start: int = 0, count: int | None = None, fanout_every: int = 4, log=None,
            out: str | None = None, save_every: int = 1) -> dict:
    """Features and plain-engine timings (ms) of every variant for instances
    [start, start + count).  With `out`, the rows collected so far are saved
    every `save_every` instances and the index being measured is written to
    `out`.progress, so a run cut short keeps its data and shows where it
    stopped."""
    import torch
    gx = _gx()
    log = log or (lambda m: print(m, flush=True))
    stop = len(instances) if count is None else min(len(instances), start + count)
    index, feats, times, ftimes, heur = [], [], [], [], []
    phase = {"make": 0.0, "features": 0.0, "variants": 0.0, "fanouts": 0.0, "heuristic": 0.0}

    def clock(name, t0):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        phase[name] += t1 - t0
        if out:
            Path(str(out) + ".progress").write_text(f"{idx} after {name}\n")
        return t1

    for idx in range(start, stop):
        inst = instances[idx]
        if out:
            Path(str(out) + ".progress").write_text(f"{idx} start\n")
        t0 = time.perf_counter()
        k, v, cdf = make_instance(inst)
        reqs = AGGS[inst.get("aggs", "sumcount")]
        t0 = clock("make", t0)
        f = features(k, v, reqs)
        t0 = clock("features", t0)
        row = []
        for algo in (gx.HASH, gx.SORT, gx.PARTITION):
            if out:
                Path(str(out) + ".progress").write_text(f"{idx} variant {algo}\n")
            row.append(time_call(lambda: gx.groupby([k], v, reqs, gx.make_hint(algo))))
        t0 = clock("variants", t0)
        fr = [np.nan] * len(FANOUTS)
        if idx % fanout_every == 0:
            for j, bits in enumerate(FANOUTS):
                if out:
                    Path(str(out) + ".progress").write_text(f"{idx} fanout {bits}\n")
                fr[j] = time_call(lambda: gx.groupby([k], v, reqs, gx.make_hint(gx.PARTITION, radix_bits=bits)))
        t0 = clock("fanouts", t0)
        h = heuristic_algo(k)
        clock("heuristic", t0)
        del k, v, cdf
        index.append(idx), feats.append(f), times.append(row), ftimes.append(fr), heur.append(h)
        if len(index) % 16 == 0:
            log(f"{idx + 1} at {time.strftime('%H:%M:%S')}: " + " ".join(f"{n}={s:.1f}s" for n, s in phase.items()))
        if out and len(index) % save_every == 0:
            np.savez(out, **_pack(instances, index, feats, times, ftimes, heur))
    data = _pack(instances, index, feats, times, ftimes, heur)
    if out:
        np.savez(out, **data)
    return data


def merge(paths: list[str]) -> dict:
    """Concatenate collected chunks in instance order (duplicates dropped)."""
    parts = [np.load(p) for p in paths]
    index = np.concatenate([d["index"] for d in parts])
    order = np.argsort(index, kind="stable")
    keep = order[np.concatenate([[True], np.diff(index[order]) != 0])] if len(order) else order
    insts = sum((json.loads(str(d["instances"])) for d in parts), [])
    out = {"index": index[keep], "instances": json.dumps([insts[i] for i in keep])}
    for key in ("features", "times", "fanout_times", "heuristic"):
        out[key] = np.concatenate([d[key] for d in parts])[keep]
    return out


def targets_from(times: np.ndarray, ftimes: np.ndarray):
    """log2 of the timings; unmeasured fan-outs are masked out."""
    t = np.zeros((times.shape[0], O), np.float32)
    m = np.zeros_like(t)
    t[:, :NV] = np.log2(times)
    m[:, :NV] = 1
    ok = ~np.isnan(ftimes)
    t[:, NV:][ok] = np.log2(ftimes[ok])
    m[:, NV:][ok] = 1
    return t, m


def train(x: np.ndarray, t: np.ndarray, m: np.ndarray, epochs: int = 1500, lr: float = 3e-3, seed: int = 0):
    """Full-batch Adam on the GPU with the library kernels; returns FP16 params."""
    import torch
    gx = _gx()
    n = param_count()
    rng = np.random.default_rng(seed)
    w = []
    for fan_in, fan_out in ((F, H), (H, H), (H, O)):
        w.append(rng.normal(0, math.sqrt(2.0 / fan_in), size=(fan_out, fan_in)).reshape(-1))
        w.append(np.zeros(fan_out))
    master = torch.from_numpy(np.concatenate(w).astype(np.float32)).cuda()
    assert master.numel() == n
    params = master.half()
    grads = torch.zeros(n, dtype=torch.float32, device="cuda")
    mom = torch.zeros_like(grads)
    vel = torch.zeros_like(grads)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    dx = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    dt = torch.from_numpy(np.ascontiguousarray(t, np.float32)).cuda()
    dm = torch.from_numpy(np.ascontiguousarray(m, np.float32)).cuda()
    s = gx._stream_ptr(None)
    hist = []
    for step in range(1, epochs + 1):
        gx.check(gx.lib.gx_mlp_forward_backward(params.data_ptr(), dx.data_ptr(), dt.data_ptr(), dm.data_ptr(),
                                                x.shape[0], grads.data_ptr(), loss.data_ptr(), s))
        gx.check(gx.lib.gx_mlp_adam_step(master.data_ptr(), params.data_ptr(), grads.data_ptr(), mom.data_ptr(),
                                         vel.data_ptr(), step, C.c_float(lr), s))
        if step % 100 == 0 or step == 1:
            hist.append((step, float(loss.item())))
    return params.cpu().numpy().view(np.uint16), hist


def predict(params_u16: np.ndarray, x: np.ndarray) -> np.ndarray:
    import torch
    gx = _gx()
    p = torch.from_numpy(params_u16.view(np.float16).copy()).cuda()
    dx = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    out = torch.empty((x.shape[0], O), dtype=torch.float32, device="cuda")
    gx.check(gx.lib.gx_mlp_forward(p.data_ptr(), dx.data_ptr(), x.shape[0], out.data_ptr(), gx._stream_ptr(None)))
    return out.cpu().numpy()


def regret(times: np.ndarray, choice: np.ndarray) -> float:
    best = times.min(axis=1)
    chosen = times[np.arange(len(choice)), choice]
    return float(np.mean(chosen / best - 1.0))


def heuristic_choice(heur_algo: np.ndarray) -> np.ndarray:
    gx = _gx()
    return np.where(heur_algo == gx.HASH, 0, np.where(heur_algo == gx.SORT, 1, 2))


def save(path: Path, params_u16: np.ndarray, mean: np.ndarray, std: np.ndarray, meta: dict) -> None:
    np.savez(path, params=params_u16, mean=mean.astype(np.float32), std=std.astype(np.float32),
             meta=json.dumps(meta), version=1)


# How far (largest difference of one plan feature) a request list may lie
# from a trained one for AUTO to trust the network: SUM + COUNT over an int32
# column (0.125 from the int64 training list) stays inside; SUM over a
# float64 column, or an extra accumulator class, does not.
SUPPORT_RADIUS = 0.13


def training_plan_support() -> np.ndarray:
    """Plan features (16..19) of the request lists in AGGS, over the value
    columns make_instance builds (int64, then float64), computed by the
    library on the host: one row per list."""
    gx = _gx()
    cols = [gx.ColumnView(None, 0, gx.INT64, 0), gx.ColumnView(None, 0, gx.FLOAT64, 0)]
    rows = []
    for reqs in AGGS.values():
        ncols = max(c for c, _ in reqs) + 1
        rows.append(plan_features(cols[:ncols], reqs))
    return np.ascontiguousarray(np.stack(rows), np.float32)


def install(path: Path | None = None) -> bool:
    """Load trained weights into the library (AUTO + hint.selector=LEARNED),
    with the request lists they were trained on as the network's support."""
    gx = _gx()
    path = Path(path) if path else WEIGHTS
    if not path.exists():
        return False
    d = np.load(path)
    p = np.ascontiguousarray(d["params"], np.uint16)
    if p.size != param_count() or d["mean"].size != F:
        return False  # weights of another network shape: keep the plain rule
    mean = np.ascontiguousarray(d["mean"], np.float32)
    std = np.ascontiguousarray(d["std"], np.float32)
    gx.check(gx.lib.gx_selector_load(p.ctypes.data, mean.ctypes.data, std.ctypes.data))
    sup = training_plan_support()
    gx.check(gx.lib.gx_selector_set_plan_support(sup.ctypes.data, len(sup), SUPPORT_RADIUS))
    return True


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--instances", type=int, default=4096)
    c.add_argument("--seed", type=int, default=7)
    c.add_argument("--out", required=True)
    c.add_argument("--start", type=int, default=0)
    c.add_argument("--count", type=int, default=None)
    mg = sub.add_parser("merge")
    mg.add_argument("chunks", nargs="+")
    mg.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("timings")
    t.add_argument("--holdout", type=int, default=1024)
    t.add_argument("--epochs", type=int, default=3000)
    t.add_argument("--out", default=str(WEIGHTS))
    t.add_argument("--report", default=None)
    t.add_argument("--heldout-out", default=None, help="save the held-out features / timings (for tests)")
    a = ap.parse_args()
    if a.cmd == "collect":
        collect(draw_instances(a.instances, a.seed), start=a.start, count=a.count, out=a.out)
        return
    if a.cmd == "merge":
        np.savez(a.out, **merge(a.chunks))
        return
    d = np.load(a.timings)
    x, times, ft = d["features"], d["times"], d["fanout_times"]
    t_all, m_all = targets_from(times, ft)
    n = x.shape[0]
    ntr = n - a.holdout
    mean, std = x[:ntr].mean(0), x[:ntr].std(0) + 1e-6
    xs = (x - mean) / std
    params, hist = train(xs[:ntr], t_all[:ntr], m_all[:ntr], epochs=a.epochs)
    y = predict(params, xs[ntr:])
    learned = np.argmin(y[:, :NV], axis=1)
    heur = heuristic_choice(d["heuristic"][ntr:])
    oracle_best = np.argmin(times[ntr:], axis=1)
    # Fan-out head: on held-out instances with measured fan-outs, the chosen
    # radix bits against the best of the four, beside a fixed 8 bits (one
    # radix pass, what the engine defaults to near 2^16 groups).
    fth = ft[ntr:]
    fok = ~np.isnan(fth).any(axis=1)
    fchoice = np.argmin(y[fok][:, NV:], axis=1)
    insts = json.loads(str(d["instances"]))[ntr:]
    kinds = np.array([i.get("aggs", "sumcount") for i in insts])
    report = {"train_instances": int(ntr), "heldout_instances": int(n - ntr),
              "regret_learned": regret(times[ntr:], learned), "regret_heuristic": regret(times[ntr:], heur),
              "accuracy_learned": float(np.mean(learned == oracle_best)),
              "accuracy_heuristic": float(np.mean(heur == oracle_best)),
              "regret_learned_by_aggs": {k: regret(times[ntr:][kinds == k], learned[kinds == k])
                                         for k in AGGS if (kinds == k).any()},
              "regret_heuristic_by_aggs": {k: regret(times[ntr:][kinds == k], heur[kinds == k])
                                           for k in AGGS if (kinds == k).any()},
              "fanout_instances": int(fok.sum()),
              "fanout_regret_learned": regret(fth[fok], fchoice) if fok.any() else None,
              "fanout_regret_fixed_8_bits": regret(fth[fok], np.zeros(int(fok.sum()), np.int64)) if fok.any() else None,
              "loss_history": hist,
              "best_variant_share": np.bincount(oracle_best, minlength=NV).tolist()}
    save(Path(a.out), params, mean, std, report)
    print(json.dumps(report))
    if a.report:
        Path(a.report).write_text(json.dumps(report, indent=1))
    if a.heldout_out:
        np.savez(a.heldout_out, features=x[ntr:], times=times[ntr:], heuristic=d["heuristic"][ntr:],
                 fanout_times=ft[ntr:], aggs=np.array([i.get("aggs", "sumcount") for i in insts]))


if __name__ == "__main__":
    main()
