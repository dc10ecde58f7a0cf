#!/usr/bin/env python
"""Benchmark of the hash GROUP BY path on B200 (one JSON line on stdout).

Default workload: the skewed single query (2^26 rows, int64 keys Zipf s=1.0
over 2^20 ids; SUM/COUNT/MIN/MAX of an int64 column and SUM of an fp32
column).  A step is one exact GROUP BY of the whole table.

  value  rows / s over K steps, inputs resident in HBM (1.34 GB > L2, so no
         flush is needed between steps), device-timed with CUDA events.
  e2e    the same through the host-buffer entry point (gba_groupby_host):
         pinned host inputs copied H2D inside every step, results read back.
  --impl reference
         the CPU restatement of the reference's algorithm (the reference has
         no CPU aggregation path) on all host cores, bounded sample per step.

Multi-GPU (torchrun): replicas only - every rank runs the same workload on its
own GPU; the time is the max over ranks; value = all rows / that time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in Path(self.path).read_text().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def get_workload(name: str):
    from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W
    return {"skewed": W.skewed, "small": W.small, "highcard": W.high_card}[name]()


def cpu_sample_rows(w) -> int:
    # about 10-30 s of single-pass CPU work over the steps of the reference arm
    return min(w.n, 1 << 24)


def run_reference(args, ws, rank):
    """The reference arm: CPU restatement of the path on all host cores."""
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import cpu_oracle as O
    from cpu_gpu_coprocess_groupby_agg_b200 import gen_host
    w = get_workload(args.workload)
    cores = os.cpu_count() or 1
    m = cpu_sample_rows(w)
    keys, cols = gen_host(w.spec, m, nthreads=cores)
    for _ in range(args.warmup):
        O.groupby(keys, cols, w.aggs, nthreads=cores, sort=False)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.groupby(keys, cols, w.aggs, nthreads=cores, sort=False)
    dt = (time.perf_counter() - t0) / args.steps
    value = m / dt / 1e9
    line = {
        "impl": "reference", "metric": "groupby_rows_per_s", "value": round(value, 6), "unit": "G rows/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded PCG32 generator)",
        "config": {"workload": w.name, "rows": w.n, "sample_rows_per_step": m, "aggs": [list(map(str, a)) for a in w.aggs]},
        "cpu_baseline": {"value": round(value, 6), "unit": "G rows/s", "cores": cores, "kind": "port",
                         "sample": f"first {m} rows of the workload per step (partitioned hash aggregation, "
                                   f"{cores} threads); the reference itself has no CPU aggregation path"},
        "e2e": {"value": round(value, 6), "unit": "G rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="skewed", choices=["skewed", "small", "highcard"])
    ap.add_argument("--sizing", default="learned", choices=["plain", "learned"])
    ap.add_argument("--no-plain-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--knob", action="append", default=[], help="name=value knob override")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_setup()

    if args.impl == "reference":
        return run_reference(args, ws, rank)

    import torch
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist

    from cpu_gpu_coprocess_groupby_agg_b200 import Context, gen_device, make_knobs
    from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
    w = get_workload(args.workload)
    ctx = Context(local)
    if args.sizing == "learned" and not E.load_default(ctx):
        raise SystemExit(f"learned sizing needs trained weights at {E.WEIGHTS}")
    keys, cols = gen_device(w.spec, w.n, device=local)
    torch.cuda.synchronize()
    kn = {"sizing": args.sizing, "timing": 1}
    for kv in args.knob:
        name, val = kv.split("=")
        kn[name] = float(val) if "." in val else int(val)
    knobs = make_knobs(**kn)
    stream = torch.cuda.current_stream()
    cap = min(w.n, max(1 << 20, w.spec.ndv * 2)) + 1
    out_keys = torch.empty(cap, dtype=keys.dtype, device=keys.device)
    out_aggs = [torch.empty(cap, dtype=torch.float64 if (op == "sum" and c is not None and w.spec.col_kind[c] == 2)
                            else torch.int64, device=keys.device) for op, c in w.aggs]

    def step():
        return ctx.groupby(keys, cols, w.aggs, knobs=knobs, out=(out_keys, out_aggs), stream=stream)

    for _ in range(args.warmup):
        res = step()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    main_ms = 0.0
    launches = 0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            res = step()
            main_ms += res.stats["kernel_ms"][1]
            launches += res.stats["kernel_launches"]
        ev1.record(stream)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    elapsed = ev0.elapsed_time(ev1)
    if pg:
        t = torch.tensor([elapsed], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        elapsed = float(t.item())
    ms_step = elapsed / args.steps
    value = ws * w.n / (ms_step / 1e3) / 1e9
    G = res.n_groups
    peak, peak_kind = peaks()
    main_avg = main_ms / args.steps
    alg_bytes = w.n * w.row_bytes()
    achieved = alg_bytes / (main_avg / 1e3) / 1e9 if main_avg > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(f"{w.name}:k_preagg")
    whole_bytes = w.n * w.row_bytes() + G * w.out_row_bytes()

    line = {
        "metric": "groupby_rows_per_s", "value": round(value, 4), "unit": "G rows/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded PCG32 generator, generated on device)",
        "config": {"workload": w.name, "rows": w.n, "groups": G, "key": f"int{w.key_bytes * 8}",
                   "aggs": [f"{op}({'*' if c is None else c})" for op, c in w.aggs], "sizing": args.sizing,
                   "strategy": res.stats["strategy"], "table_slots": res.stats["table_slots"],
                   "l2": "inputs larger than L2 (no flush needed)", "parallelism": f"replicas x{ws}"},
        "whole_step_hbm_gbs": round(whole_bytes / (ms_step / 1e3) / 1e9, 1),
        "roofline": {"bound": "hbm", "kernel": "k_preagg", "achieved": round(achieved, 1) if achieved else None,
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "alg_bytes_per_launch": alg_bytes, "launch_ms": round(main_avg, 4)},
        "gpu_launches": launches,
    }
    line["clocks"] = clk.summary()
    line["config"]["predicted_groups"] = round(res.stats["predicted_groups"], 1)

    if args.sizing == "learned" and not args.no_plain_compare:
        # the same workload with plain (estimator-free) sizing, for comparison
        pk = make_knobs(sizing="plain", timing=1)
        for _ in range(2):
            ctx.groupby(keys, cols, w.aggs, knobs=pk, out=(out_keys, out_aggs), stream=stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(2, min(args.steps, 5))
        e0.record(stream)
        for _ in range(reps):
            pres = ctx.groupby(keys, cols, w.aggs, knobs=pk, out=(out_keys, out_aggs), stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1) / reps
        line["plain_sizing"] = {"value": round(w.n / (pms / 1e3) / 1e9, 4), "unit": "G rows/s",
                                "ms_per_step": round(pms, 4), "strategy": pres.stats["strategy"],
                                "table_slots": pres.stats["table_slots"],
                                "partition_bits": pres.stats["partition_bits"]}

    if not args.no_e2e and rank == 0:
        line["e2e"] = e2e(ctx, w, keys, cols, knobs, args, ws)
    if not args.no_cpu_baseline and rank == 0 and ws == 1:
        line["cpu_baseline"] = cpu_baseline(w, keys, cols)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def e2e(ctx, w, keys, cols, knobs, args, ws):
    """Same metric through gba_groupby_host: pinned host columns in, host results out."""
    import torch
    hk = keys.cpu().pin_memory()
    hc = [c.cpu().pin_memory() for c in cols]
    hk_np = hk.numpy()
    hc_np = [c.numpy() for c in hc]
    cap = min(w.n, max(1 << 20, w.spec.ndv * 2)) + 1
    ok = torch.empty(cap, dtype=hk.dtype).pin_memory().numpy()
    oa = [torch.empty(cap, dtype=torch.float64 if (op == "sum" and c is not None and w.spec.col_kind[c] == 2)
                      else torch.int64).pin_memory().numpy() for op, c in w.aggs]
    stream = torch.cuda.current_stream()
    for _ in range(2):
        res = ctx.groupby_host(hk_np, hc_np, w.aggs, knobs=knobs, out=(ok, oa), stream=stream)
    torch.cuda.synchronize()
    steps = max(3, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(steps):
        res = ctx.groupby_host(hk_np, hc_np, w.aggs, knobs=knobs, out=(ok, oa), stream=stream)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    return {"value": round(w.n / dt / 1e9, 4), "unit": "G rows/s", "ms_per_step": round(dt * 1e3, 3),
            "h2d_bytes_per_step": w.n * w.row_bytes(),
            "d2h_bytes_per_step": res.n_groups * w.out_row_bytes(), "pinned": True,
            "timer": "host wall clock around the synchronous call"}


def cpu_baseline(w, keys, cols):
    sys.path.insert(0, str(ROOT / "oracle"))
    import cpu_oracle as O
    m = cpu_sample_rows(w)
    hk = keys[:m].cpu().numpy()
    hc = [c[:m].cpu().numpy() for c in cols]
    cores = os.cpu_count() or 1
    O.groupby(hk, hc, w.aggs, nthreads=cores, sort=False)
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        O.groupby(hk, hc, w.aggs, nthreads=cores, sort=False)
    dt = (time.perf_counter() - t0) / reps
    return {"value": round(m / dt / 1e9, 6), "unit": "G rows/s", "cores": cores, "kind": "port",
            "sample": f"first {m} rows of the workload, partitioned hash aggregation on {cores} threads, "
                      f"mean of {reps} runs"}


if __name__ == "__main__":
    sys.exit(main())
