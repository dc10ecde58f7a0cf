#!/usr/bin/env python
"""Benchmark of the hash GROUP BY path on B200 (one JSON line on stdout).

Default workload (--workload batch): the 256-query mixed batch (rows
log-uniform in [2^12, 2^24], distinct keys log-uniform in [16, rows/2], Zipf
s in [0, 1.5], int32/int64 keys 50/50, SUM + COUNT of an int64 column).  A step
is one gba_groupby_batch call over all 256 queries with learned sizing; the
same batch with plain sizing is timed beside it (plain_sizing).  Single-query
workloads: skewed (2^26 rows, int64 keys Zipf s=1.0 over 2^20 ids;
SUM/COUNT/MIN/MAX of an int64 column and SUM of an fp32 column), small,
highcard.

  value  rows / s over K steps, inputs resident in HBM (several GB > L2, so no
         flush is needed between steps), device-timed with CUDA events.
  e2e    the same through the public API with host buffers: pinned host
         inputs copied H2D inside every step, results read back.
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


def max_over_ranks(x: float, dist, device) -> float:
    """The largest x over all ranks (the job's time is its slowest rank's)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def get_workload(name: str, rows: int = 0):
    """A single-query workload; rows > 0 takes that many rows of the same
    shape (distinct ids of the high-cardinality workload scale alike), for
    profiling captures that must stay small."""
    import dataclasses
    from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W
    w = {"skewed": W.skewed, "small": W.small, "highcard": W.high_card,
         "large": lambda: W.large_serving_query(seed=900)}[name]()
    if rows > 0 and rows != w.n:
        if name == "highcard":
            w = W.high_card(n=rows, ndv=max(1, rows // 4))
        else:
            w = dataclasses.replace(w, n=rows, name=f"{w.name}[rows {rows}]")
    return w


BATCH_NAME = "batch_256q_rows2^12-2^24_logu_ndv16-rows/2_zipf0-1.5_sum+count"


def batch_cpu_sample(ws_list, limit=1 << 24):
    """Leading queries of the batch whose rows add up to about `limit`."""
    out, tot = [], 0
    for w in ws_list:
        if tot >= limit:
            break
        out.append(w)
        tot += w.n
    return out, tot


def cpu_sample_rows(w) -> int:
    # about 10-30 s of single-pass CPU work over the steps of the reference arm
    return min(w.n, 1 << 24)


def cpu_model() -> str:
    """The host CPU's model name (first /proc/cpuinfo entry)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def run_reference(args, ws, rank):
    """The reference arm: the CPU restatement of the path (the reference has no
    CPU aggregation path of its own) on all host cores.  For the batch every
    step is the WHOLE 256-query batch, the GPU arm's workload; inputs come
    from the oracle's copy of the seeded generator, so this process never
    loads the library.  A single-thread time over the batch's first queries is
    reported beside it."""
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import cpu_oracle as O
    from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W  # generator specs only; no library load
    cores = os.cpu_count() or 1
    if args.workload == "batch":
        allq = W.batch_queries()
        name = BATCH_NAME
        if args.ndv_range:
            lo, hi = (float(x) for x in args.ndv_range.split(":"))
            allq = [q for q in allq if lo <= q.meta["ndv"] < hi]
            name = f"{BATCH_NAME}[ndv {args.ndv_range}]"
        data = [O.gen(q.spec, q.n, nthreads=cores) for q in allq]
        total_rows = m = sum(q.n for q in allq)
        aggs = allq[0].aggs

        def one(threads=cores, upto=None):
            for q, (k, c) in list(zip(allq, data))[:upto]:
                O.groupby(k, c, q.aggs, nthreads=threads, sort=False)
        what = f"all {len(allq)} queries of the batch ({m} rows) per step, the GPU arm's workload"
        sample, m1 = batch_cpu_sample(allq)
        single = (len(sample), m1)
        same = True
    else:
        w = get_workload(args.workload, args.rows)
        m = cpu_sample_rows(w)
        keys, cols = O.gen(w.spec, m, nthreads=cores)
        name, total_rows, aggs = w.name, w.n, w.aggs

        def one(threads=cores, upto=None):
            O.groupby(keys, cols, w.aggs, nthreads=threads, sort=False)
        what = f"first {m} rows of the workload per step"
        single = (1, m)
        same = m == w.n
    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    dt = (time.perf_counter() - t0) / args.steps
    value = m / dt / 1e9
    # one thread, over a bounded sample (the leading queries of the batch)
    t1 = time.perf_counter()
    one(threads=1, upto=single[0])
    st_value = single[1] / (time.perf_counter() - t1) / 1e9
    line = {
        "impl": "reference", "metric": "groupby_rows_per_s", "value": round(value, 6), "unit": "G rows/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded PCG32 generator; the oracle's copy, bit-identical to the GPU arm's)",
        "config": {"workload": name, "rows": total_rows, "rows_per_step": m, "same_config": same,
                   "aggs": [list(map(str, a)) for a in aggs]},
        "cpu_baseline": {"value": round(value, 6), "unit": "G rows/s", "cores": cores, "kind": "port",
                         "cpu_model": cpu_model(),
                         "sample": f"{what} (partitioned hash aggregation, {cores} threads); the reference "
                                   f"itself has no CPU aggregation path",
                         "single_thread": {"value": round(st_value, 6), "unit": "G rows/s", "cores": 1,
                                           "sample": f"the first {single[0]} queries ({single[1]} rows), one pass"}},
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
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "skewed", "small", "highcard", "large", "serve", "dropin"])
    ap.add_argument("--duration", type=float, default=10.0, help="serve: seconds of Poisson arrivals")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: arrivals per second")
    ap.add_argument("--max-inflight", type=int, default=256, help="serve: client-side cap on requests in flight")
    ap.add_argument("--sizing", default="learned", choices=["plain", "learned"])
    ap.add_argument("--no-plain-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--knob", action="append", default=[], help="name=value knob override")
    ap.add_argument("--no-autotune", action="store_true", help="batch: default knobs instead of gba_autotune's")
    ap.add_argument("--ndv-range", default="", help="batch: only queries with LO <= distinct ids < HI ('LO:HI')")
    ap.add_argument("--rows", type=int, default=0, help="single query: rows of a smaller case of the same shape")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_setup()

    if args.impl == "reference":
        return run_reference(args, ws, rank)
    if args.workload == "dropin":
        return run_dropin(args, ws, rank)

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
    if args.workload == "batch":
        return run_batch(args, ws, rank, local, pg)
    if args.workload == "serve":
        return run_serve(args, ws, rank, local, pg)
    w = get_workload(args.workload, args.rows)
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
        elapsed = max_over_ranks(elapsed, pg, "cuda")
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
        traffic = json.loads(tfile.read_text()).get(
            f"{w.name}:{'k_part_agg' if res.stats['strategy'] == 2 else 'k_preagg'}")
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
        "roofline": {"bound": "hbm", "kernel": "k_part_agg" if res.stats["strategy"] == 2 else "k_preagg",
                     "achieved": round(achieved, 1) if achieved else None,
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


def _knob_overrides(args) -> dict:
    kn = {}
    for kv in args.knob:
        name, val = kv.split("=")
        kn[name] = float(val) if "." in val else int(val)
    return kn


def run_batch(args, ws, rank, local, pg):
    """The 256-query mixed batch in one gba_groupby_batch call per step."""
    import torch
    from cpu_gpu_coprocess_groupby_agg_b200 import Context, gen_device, make_knobs
    from cpu_gpu_coprocess_groupby_agg_b200 import _abi as A
    from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
    from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W
    allq = W.batch_queries()
    name = BATCH_NAME
    if args.ndv_range:
        # a slice of the batch by distinct ids (profiling one cardinality class)
        lo, hi = (float(x) for x in args.ndv_range.split(":"))
        allq = [q for q in allq if lo <= q.meta["ndv"] < hi]
        name = f"{BATCH_NAME}[ndv {args.ndv_range}]"
    ctx = Context(local)
    if args.sizing == "learned" and not E.load_default(ctx):
        raise SystemExit(f"learned sizing needs trained weights at {E.WEIGHTS}")
    dq = []
    for q in allq:
        k, c = gen_device(q.spec, q.n, device=local)
        dq.append((k, c, q.aggs))
    torch.cuda.synchronize()
    total_rows = sum(q.n for q in allq)
    in_bytes = sum(q.n * q.row_bytes() for q in allq)
    outs = ctx.batch_outputs(dq)
    stream = torch.cuda.current_stream()
    base = {"timing": 1}
    base.update(_knob_overrides(args))
    # knobs per sizing: the autotuner's choice on this batch (outside the timed
    # region), unless --no-autotune or knob overrides are given
    tuned = {}

    def knobs_for(sizing):
        if sizing in tuned:
            return tuned[sizing][0]
        kn = make_knobs(**dict(base, sizing=sizing))
        if not args.no_autotune and not args.knob:
            best, ms = ctx.autotune(dq, knobs=kn, outs=outs, stream=stream)
            best.timing = 1
            tuned[sizing] = (best, ms)
            return best
        tuned[sizing] = (kn, None)
        return kn

    def knob_summary(k):
        return {"use_tma": k.use_tma, "nstages": k.nstages, "coalesce": k.coalesce,
                "blocks_per_sm": k.blocks_per_sm, "block_threads": k.block_threads,
                "learned_load": k.learned_load, "load_factor": k.load_factor,
                "item_rows": k.item_rows, "smem_probe_cap": k.smem_probe_cap, "table_slots": k.table_slots}

    pb = ctx.prepare_batch(dq, outs)

    def timed(sizing, steps, clocks=False):
        # the steps run with the library's defaults (no per-kernel events: with
        # them the batch also runs its table clears and compactions apart from
        # the streaming launches); a second pass of as many steps with kernel
        # timing on gives the streaming launches' own time for the roofline
        knobs_t = knobs_for(sizing)
        knobs = A.Knobs.from_buffer_copy(knobs_t)
        knobs.timing = 0
        for _ in range(args.warmup):
            ctx.run_batch(pb, knobs=knobs, stream=stream)
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        main_ms, main_bytes, launches = 0.0, 0, 0
        with ClockSampler(local) as clk:
            e0.record(stream)
            for _ in range(steps):
                ng = ctx.run_batch(pb, knobs=knobs, stream=stream)
                st = ctx.stats()
                main_bytes += st["main_bytes"]
                launches += st["kernel_launches"]
            e1.record(stream)
            torch.cuda.synchronize()
        if pg:
            pg.barrier()
        el = e0.elapsed_time(e1)
        if pg:
            el = max_over_ranks(el, pg, "cuda")
        ctx.run_batch(pb, knobs=knobs_t, stream=stream)  # (a new launch graph)
        for _ in range(steps):
            ctx.run_batch(pb, knobs=knobs_t, stream=stream)
            main_ms += ctx.stats()["kernel_ms"][1]
        torch.cuda.synchronize()
        return el / steps, main_ms / steps, main_bytes / steps, launches, (ng, st), clk.summary()

    ms_step, main_ms, main_bytes, launches, res, clocks = timed(args.sizing, args.steps)
    value = ws * total_rows / (ms_step / 1e3) / 1e9
    ng, st = res
    groups = int(ng.sum())
    peak, peak_kind = peaks()
    achieved = main_bytes / (main_ms / 1e3) / 1e9 if main_ms > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get(f"{name}:k_stream_agg")
    line = {
        "metric": "groupby_rows_per_s", "value": round(value, 4), "unit": "G rows/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded PCG32 generator, generated on device)",
        "config": {"workload": name, "queries": len(allq), "rows": total_rows, "input_bytes": in_bytes,
                   "groups": groups, "aggs": ["sum(0)", "count(*)"], "sizing": args.sizing,
                   "strategy_mix": st["strategy"], "table_slots_total": st["table_slots"],
                   "predicted_groups_total": round(st["predicted_groups"], 1),
                   "l2": "inputs larger than L2 (no flush needed)", "parallelism": f"replicas x{ws}",
                   "launch": "one gba_groupby_batch call per step (CUDA graph replay)",
                   "knobs": knob_summary(tuned[args.sizing][0]),
                   "knobs_from": "gba_autotune on this batch before timing" if tuned[args.sizing][1] is not None
                   else "defaults / --knob"},
        "whole_step_hbm_gbs": round(in_bytes / (ms_step / 1e3) / 1e9, 1),
        "roofline": {"bound": "hbm",
                     "kernel": "k_stream_agg + k_stream_tma (the batch's streaming launches; + k_part_agg of "
                               "partition-strategy queries)",
                     "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None, "peak_kind": peak_kind,
                     "traffic": traffic, "alg_bytes_per_step": int(main_bytes), "launch_ms": round(main_ms, 4)},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if args.sizing == "learned" and not args.no_plain_compare:
        # the estimator-free methods on the same batch: tables sized by the row
        # count ("plain"), and tables that start at most 2^16 slots and regrow
        # 4x on overflow ("grow"); the speed-up is against the faster of them
        alt = {}
        for sz in ("plain", "grow"):
            pms, pmain, pbytes, _, pres, _ = timed(sz, max(3, min(args.steps, 5)))
            alt[sz] = {"value": round(ws * total_rows / (pms / 1e3) / 1e9, 4), "unit": "G rows/s",
                       "ms_per_step": round(pms, 4), "strategy_mix": pres[1]["strategy"],
                       "table_slots_total": pres[1]["table_slots"], "regrows": pres[1]["regrows"],
                       "knobs": knob_summary(tuned[sz][0])}
        fastest = min(alt, key=lambda z: alt[z]["ms_per_step"])
        line["plain_sizing"] = dict(alt["plain"], grow=alt["grow"], faster=fastest,
                                    learned_speedup=round(alt[fastest]["ms_per_step"] / ms_step, 3))
    if not args.no_e2e and rank == 0:
        line["e2e"] = batch_e2e(ctx, allq, dq, outs, knobs_for(args.sizing), args)
    if not args.no_cpu_baseline and rank == 0 and ws == 1:
        # the oracle over the whole batch (one pass, all host cores), and on
        # one thread over the batch's leading queries
        sys.path.insert(0, str(ROOT / "oracle"))
        import cpu_oracle as O
        host = [(k.cpu().numpy(), [c.cpu().numpy() for c in cs]) for k, cs, _ in dq]
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        for (k, c), q in zip(host, allq):
            O.groupby(k, c, q.aggs, nthreads=cores, sort=False)
        dt = time.perf_counter() - t0
        sample, m1 = batch_cpu_sample(allq)
        t1 = time.perf_counter()
        for (k, c), q in zip(host, sample):
            O.groupby(k, c, q.aggs, nthreads=1, sort=False)
        dt1 = time.perf_counter() - t1
        del host
        line["cpu_baseline"] = {"value": round(total_rows / dt / 1e9, 6), "unit": "G rows/s", "cores": cores,
                                "kind": "port", "cpu_model": cpu_model(),
                                "sample": f"all {len(allq)} queries ({total_rows} rows), one pass, partitioned "
                                          f"hash aggregation on {cores} threads",
                                "single_thread": {"value": round(m1 / dt1 / 1e9, 6), "unit": "G rows/s", "cores": 1,
                                                  "sample": f"the first {len(sample)} queries ({m1} rows), one pass"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del outs, dq
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


DROPIN_CASES = [  # name, seed, rows, distinct keys, tile_len, P, nstreams
    ("small_2^20_uniform_1024", 1, 1 << 20, 1024, 1 << 18, 300, 4),
    ("u32_2^26_uniform_2^20", 31, 1 << 26, 1 << 20, 1 << 22, 300, 4),
]


def run_dropin(args, ws, rank):
    """The reference's own GPU path against this library's C++ drop-in, on the
    same pinned u32 input and the same call sequence (test/test.cu:134-161:
    groupby_agg_partition, then groupby_agg_intra_partition with
    min/max_load_num = 3/5, 4/5 of Capacity = tile_len): oracle/_ref/ref_driver
    is the unmodified reference built from its sources, lib/tiled_driver links
    libgba.so through include/tiled_groupby_agg_partition.hpp.  Both are
    host-resident end to end (PCIe included).  Each driver runs both phases
    `steps` times in one process; the first run is a warm-up."""
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import cpu_oracle as O
    from cpu_gpu_coprocess_groupby_agg_b200.api import gen_spec  # pure Python spec; no library load
    drivers = {"reference": ROOT / "oracle" / "_ref" / "ref_driver",
               "dropin": ROOT / "cpu_gpu_coprocess_groupby_agg_b200" / "lib" / "tiled_driver"}
    reps = max(3, args.steps)
    rows = {}
    with tempfile.TemporaryDirectory() as td:
        for name, seed, n, ndv, tile, P, ns in DROPIN_CASES:
            sp = gen_spec(seed, 32, ndv, 0.0, [("i32", 0, 1000)], permute_ids=True, avoid_all_ones=True)
            keys, cols = O.gen(sp, n, nthreads=os.cpu_count() or 1, key_unsigned=True)
            inp = Path(td) / f"{name}.in"
            with open(inp, "wb") as f:
                f.write(np.int64(n).tobytes())
                f.write(keys.astype(np.uint32).tobytes())
                f.write(cols[0].astype(np.uint32).tobytes())
            case = {"rows": n, "distinct_keys": ndv, "tile_len": tile, "P": P, "nstreams": ns}
            for who, exe in drivers.items():
                if not exe.exists():
                    case[who] = {"unavailable": f"{exe.name} not built"}
                    continue
                outp = Path(td) / f"{name}.{who}"
                r = subprocess.run([str(exe), str(inp), str(outp), str(tile), str(P), str(ns), str(tile), str(reps)],
                                   capture_output=True, text=True, timeout=1200)
                if r.returncode != 0:
                    case[who] = {"unavailable": f"exit {r.returncode}: {r.stderr.strip()[-200:]}"}
                    continue
                meta = json.loads(Path(str(outp) + ".json").read_text())
                tot = [a + b for a, b in zip(meta["phase1_s_all"], meta["phase2_s_all"])][1:]
                t = statistics.median(tot)
                case[who] = {"value": round(n / t / 1e9, 4), "unit": "G rows/s", "ms": round(t * 1e3, 3),
                             "phase1_ms": round(statistics.median(meta["phase1_s_all"][1:]) * 1e3, 3),
                             "phase2_ms": round(statistics.median(meta["phase2_s_all"][1:]) * 1e3, 3),
                             "runs": len(tot), "groups": int(sum(meta["par_result_kv_num"]))}
            if "value" in case.get("reference", {}) and "value" in case.get("dropin", {}):
                case["speedup"] = round(case["dropin"]["value"] / case["reference"]["value"], 2)
                case["same_groups"] = case["dropin"]["groups"] == case["reference"]["groups"]
            rows[name] = case
    big = rows[DROPIN_CASES[-1][0]]
    value = big.get("dropin", {}).get("value")
    line = {"metric": "groupby_rows_per_s", "value": value, "unit": "G rows/s", "n_gpus": 1, "steps": reps - 1,
            "warmup": 1, "ms_per_step": big.get("dropin", {}).get("ms"), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded PCG32 generator), pinned host memory",
            "config": {"workload": "dropin_vs_reference_gpu", "cases": rows,
                       "timer": "host steady_clock inside each driver, both phases, median of the runs after the "
                                "first"}}
    print(json.dumps(line), flush=True)
    return 0


SERVE_NAME = "serve_poisson_batch256shapes+5%_2^27rows_2^24keys"


def run_serve(args, ws, rank, local, pg):
    """Serving stream: Poisson arrivals of queries drawn from the 256-query
    batch's shapes, plus 5% large queries (2^27 rows over 2^24 int64 ids), into
    a gba_server with a 120 GiB budget; inputs device-resident.  Reported: the
    sustained rows/s (rows of finished requests / time from the first arrival
    to the last completion) and p50/p99 latency, learned and plain sizing.
    Timing is host wall clock (a latency is submit -> result on the device)."""
    import numpy as np
    import torch
    from cpu_gpu_coprocess_groupby_agg_b200 import Server, gen_device, make_knobs
    from cpu_gpu_coprocess_groupby_agg_b200 import estimator as E
    from cpu_gpu_coprocess_groupby_agg_b200 import workloads as W
    small = W.batch_queries()
    large = [W.large_serving_query(seed=900 + i) for i in range(2)]
    pool = small + large
    data = []
    for q in pool:
        k, c = gen_device(q.spec, q.n, device=local)
        data.append((k, c, q.aggs))
    torch.cuda.synchronize()
    free = [[] for _ in pool]

    def out_for(i):
        if free[i]:
            return free[i].pop()
        q = pool[i]
        cap = min(q.n, q.spec.ndv) + 1
        return (torch.empty(cap, dtype=data[i][0].dtype, device=data[i][0].device),
                [torch.empty(cap, dtype=torch.int64, device=data[i][0].device) for _ in q.aggs])

    def one_run(sizing, seed):
        rng = np.random.default_rng(seed)
        n_arr = int(args.rate * args.duration)
        gaps = rng.exponential(1.0 / args.rate, n_arr)
        kinds = np.where(rng.random(n_arr) < 0.05, rng.integers(len(small), len(pool), n_arr),
                         rng.integers(0, len(small), n_arr))
        sv = Server(local, lanes=4, memory_budget=120 << 30, max_batch=64, batch_rows=1 << 24,
                    knobs=make_knobs(sizing=sizing),
                    estimator_params=E.load_weights() if sizing == "learned" else None)
        inflight = {}
        infos = []

        def collect(timeout):
            info = sv.next_done(timeout)
            while info is not None:
                i, o, lag = inflight.pop(info.ticket)
                free[i].append(o)
                infos.append((info, pool[i].n, lag))
                info = sv.next_done(0.0)
        t0 = time.perf_counter()
        t_next = t0
        for j in range(n_arr):
            t_next += gaps[j]
            while True:
                now = time.perf_counter()
                if now >= t_next and len(inflight) < args.max_inflight:
                    break
                collect(min(0.002, max(t_next - now, 0.0005)))
            i = int(kinds[j])
            o = out_for(i)
            t = sv.submit(data[i][0], data[i][1], data[i][2], o)
            # a request held back by the client's in-flight cap waits from its
            # scheduled arrival: that wait is part of its latency
            inflight[t] = (i, o, (time.perf_counter() - t_next) * 1e3)
        while inflight:
            collect(1.0)
        t_end = time.perf_counter()
        err = sv._lib.gba_server_last_error(sv._h).decode()
        counters = sv.counters()
        sv.close()
        bad = [x for x, _, _ in infos if x.status != 0]
        if bad:
            raise SystemExit(f"serving: {len(bad)} requests failed, first status {bad[0].status}: {err}")
        lat = np.array([x.latency_ms + lag for x, _, lag in infos])
        rows = sum(n for _, n, _ in infos)
        big = np.array([n >= (1 << 27) for _, n, _ in infos])
        svc = np.array([x.service_ms for x, _, _ in infos])

        def pct(a, q):
            return round(float(np.percentile(a, q)), 3) if len(a) else None
        return {"value": round(rows / (t_end - t0) / 1e9, 4), "unit": "G rows/s", "requests": len(infos),
                "last_error": err,
                "seconds": round(t_end - t0, 3), "offered_seconds": round(float(np.sum(gaps)), 3),
                "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "mean_batch": round(float(np.mean([x.batch_size for x, _, _ in infos])), 2),
                "service_p99_ms": pct(svc, 99), "server": counters,
                "large_requests": {"count": int(big.sum()), "p50_ms": pct(lat[big], 50), "p99_ms": pct(lat[big], 99),
                                   "service_p50_ms": pct(svc[big], 50)},
                "small_requests": {"count": int((~big).sum()), "p50_ms": pct(lat[~big], 50),
                                   "p99_ms": pct(lat[~big], 99), "service_p50_ms": pct(svc[~big], 50)}}

    learned = one_run("learned", 5)
    plain = one_run("plain", 5)
    line = {
        "metric": "groupby_rows_per_s", "value": learned["value"], "unit": "G rows/s", "n_gpus": ws,
        "steps": learned["requests"], "warmup": 0, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded PCG32 generator, generated on device)",
        "config": {"workload": SERVE_NAME, "rate_per_s": args.rate, "duration_s": args.duration, "lanes": 4,
                   "max_inflight": args.max_inflight,
                   "latency": "scheduled arrival -> result complete (client-side wait included)",
                   "memory_budget_gib": 120, "max_batch": 64, "sizing": "learned",
                   "timer": "host wall clock, first arrival to last completion"},
        "latency_ms": {"p50": learned["p50_ms"], "p99": learned["p99_ms"]},
        "serve": learned, "plain_sizing": plain,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def batch_e2e(ctx, allq, dq, outs, knobs, args):
    """The batch through gba_groupby_batch_host, the call a user with
    host-resident data makes: pinned host columns in, pinned host groups out.
    The library cuts the batch into parts and overlaps each part's copies with
    the previous part's aggregation and the groups' copies back."""
    import numpy as np
    import torch
    npdt = {torch.int64: np.int64, torch.float64: np.float64}
    hq = []
    for q in dq:
        keys, cols, aggs = q[0], q[1], q[2]
        uk = q[3] if len(q) > 3 else False
        uc = list(q[4]) if len(q) > 4 else [False] * len(cols)
        hk = keys.cpu().pin_memory().numpy()
        hk = hk.view(np.uint32) if uk else hk
        hc = [c.cpu().pin_memory().numpy() for c in cols]
        hc = [c.view(np.uint32) if u else c for c, u in zip(hc, uc)]
        hq.append((hk, hc, aggs))
    first = ctx.groupby_batch(dq, knobs=knobs, outs=outs)

    def pinned(n, dt):
        return torch.empty(n * np.dtype(dt).itemsize, dtype=torch.uint8).pin_memory().numpy().view(dt)

    hout = [(pinned(r.n_groups + 1, hk.dtype), [pinned(r.n_groups + 1, npdt[a.dtype]) for a in oa])
            for r, (hk, _, _), (_, oa) in zip(first, hq, outs)]
    h2d = sum(k.nbytes + sum(c.nbytes for c in cs) for k, cs, _ in hq)
    stream = torch.cuda.current_stream()

    def step():
        res = ctx.groupby_batch_host(hq, hout, knobs=knobs, stream=stream)
        return sum(r.n_groups * (r.keys.itemsize + 8 * len(r.aggs)) for r in res)

    for _ in range(2):
        step()
    steps = max(3, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(steps):
        d2h = step()
    dt = (time.perf_counter() - t0) / steps
    total = sum(q.n for q in allq)
    return {"value": round(total / dt / 1e9, 4), "unit": "G rows/s", "ms_per_step": round(dt * 1e3, 3),
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "pinned": True,
            "api": "gba_groupby_batch_host",
            "timer": "host wall clock around the call (copies in, aggregation, copies out)"}


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
    m1 = min(m, 1 << 22)
    t1 = time.perf_counter()
    O.groupby(hk[:m1], [c[:m1] for c in hc], w.aggs, nthreads=1, sort=False)
    dt1 = time.perf_counter() - t1
    return {"value": round(m / dt / 1e9, 6), "unit": "G rows/s", "cores": cores, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"first {m} rows of the workload, partitioned hash aggregation on {cores} threads, "
                      f"mean of {reps} runs",
            "single_thread": {"value": round(m1 / dt1 / 1e9, 6), "unit": "G rows/s", "cores": 1,
                              "sample": f"first {m1} rows, one pass"}}


if __name__ == "__main__":
    sys.exit(main())
