#!/usr/bin/env python
"""Headline benchmark: edge updates/sec and incremental matches/sec of the
per-batch GPU pipeline (index update + delta lists + merged matching) on the
R-MAT 1M-vertex / 10M-edge stream (batches of 100,000 insertions, 9-vertex
dense pattern), with p50/p99 per-batch latency.

A step is one batch through the hot path.  The stream has 10 batches; steps
cycle through them, rebuilding the initial index (untimed) when the cycle
restarts, so every cycle sees identical work.

  value  keys already resident in HBM; time = sum of per-step device
         intervals (CUDA events on the engine's stream), max over ranks
  e2e    the same batches through the C-ABI call with host buffers
         (cgb_apply_batch: H2D of the keys, compute, D2H of the count)
Stage 1 (the CaLiG producer that makes the keys) runs before timing.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 run under torchrun: every rank keeps a full index replica and
applies every batch; the matching of each batch is split by seed (rank r
expands delta edges i with i % N == r); counts are summed and step times
maxed over ranks (NCCL).  Total work per batch is fixed: scaling "strong".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profiled_traffic(kernel: str):
    """DRAM bytes (read + write) of one launch of `kernel` on this workload, from
    the committed ncu summary (profiles/<kernel>_rmat1m10m.md, a line
    "traffic_bytes_per_launch: N"); None when there is no such capture."""
    import re

    path = os.path.join(ROOT, "profiles", f"{kernel}_rmat1m10m.md")
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*(\d+)", open(path).read())
        return (int(m.group(1)), os.path.relpath(path, ROOT)) if m else (None, None)
    except OSError:
        return None, None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"cgb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                t = [x.strip() for x in line.split(",")]
                if len(t) >= 9:
                    rows.append(t)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def log(msg: str) -> None:
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def setup_workload(rank: int):
    from cgbdsm_b200 import Producer
    from cgbdsm_b200.workloads import SPECS, materialize, read_query

    spec = SPECS[WORKLOAD]
    log(f"generating workload {spec.name}")
    paths = materialize(spec, os.environ.get("CGB_BENCH_DIR", f"/tmp/cgb_bench_r{rank}"))
    log("stage 1 (CaLiG producer) for every batch")
    t0 = time.perf_counter()
    prod = Producer(paths["query"], paths["data"], paths["update"], spec.cli_batch_size)
    init, dv0 = prod.initial()
    batches = [prod.next() for _ in range(prod.num_batches)]
    s1_s = time.perf_counter() - t0
    log(f"stage 1 done in {s1_s:.1f} s: {len(init)} initial keys, {len(batches)} batches")
    ql, qe = read_query(paths["query"])
    prod.close()
    return spec, paths, ql, qe, init, dv0, batches, s1_s


def run_ours(args) -> None:
    import torch

    from cgbdsm_b200 import Engine, dist

    rank, world, local = dist.env()
    torch.cuda.set_device(local)
    dist.init("nccl", timeout_s=600)

    spec, paths, ql, qe, init, dv0, batches, s1_s = setup_workload(rank)
    nb = len(batches)

    def new_engine():
        e = Engine(device=local, dfs_budget_ms=args.budget_ms, shard_index=rank, num_shards=world)
        e.load_query(len(ql), qe, ql)
        e.build_index(init, dv0)
        return e

    # device-resident keys per batch: [ins | del | delta]
    dev = []
    for b in batches:
        cat = np.concatenate([b["ins"], b["del"], b["delta"]]).view(np.int64)
        t = torch.from_numpy(cat).to(f"cuda:{local}")
        dev.append((t, len(b["ins"]), len(b["del"]), len(b["delta"])))
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f"cuda:{local}")
    torch.cuda.synchronize()

    eng = new_engine()
    state = {"eng": eng, "pos": 0}

    def one_step(device_keys: bool):
        if state["pos"] == nb:  # restart the stream: fresh index (untimed)
            state["eng"].close()
            state["eng"] = new_engine()
            state["pos"] = 0
        b = state["pos"]
        e = state["eng"]
        l0 = e.kernel_launches()
        if device_keys:
            flush.zero_()  # evict L2 between steps (outside the engine's timed interval)
            torch.cuda.synchronize()
            t, ni, nd, nD = dev[b]
            base = t.data_ptr()
            c = e.apply_batch_device(batches[b]["dv"], base, ni, base + 8 * ni, nd, base + 8 * (ni + nd), nD)
            ms = float(e.timings()[3])
        else:
            bb = batches[b]
            t0 = time.perf_counter()
            c = e.apply_batch(bb["dv"], bb["ins"], bb["del"], bb["delta"], bb["edge_ok"])
            ms = (time.perf_counter() - t0) * 1e3
        tm = e.timings()
        st = e.stats()
        st["launches"] = e.kernel_launches() - l0
        state["pos"] += 1
        log(f"batch {b} ({'device' if device_keys else 'host'} keys): {ms:.1f} ms, count {c}, "
            f"phases {[round(float(x), 2) for x in tm[:3]]}")
        return b, c, ms, tm, st

    for _ in range(args.warmup):
        one_step(True)
    dist.barrier()
    torch.cuda.synchronize()
    recs = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            recs.append(one_step(True))
    torch.cuda.synchronize()
    dist.barrier()
    launches = sum(r[4]["launches"] for r in recs)

    step_ms = dist.max_values([r[2] for r in recs])          # max over ranks, per step
    counts = dist.sum_counts([int(r[1]) for r in recs])       # shard counts summed, per step
    total_ms = sum(step_ms)
    edges = sum(batches[r[0]]["num_edges"] for r in recs)     # every rank sees the same batches
    matches = sum(counts)

    # e2e through the host-buffer C-ABI call (same batches, same cycle)
    state["eng"].close()
    state["eng"] = new_engine()
    state["pos"] = 0
    if args.quick:
        e2e_recs = recs
    else:
        for _ in range(args.warmup):
            one_step(False)
        e2e_recs = [one_step(False) for _ in range(args.steps)]
    e2e_ms = sum(dist.max_values([r[2] for r in e2e_recs]))
    e2e_edges = sum(batches[r[0]]["num_edges"] for r in e2e_recs)
    h2d = sum(8 * (len(batches[r[0]]["ins"]) + len(batches[r[0]]["del"]) + len(batches[r[0]]["delta"]))
              + len(batches[r[0]]["edge_ok"]) for r in e2e_recs) / len(e2e_recs)

    # roofline of the dominant kernel (by time over the timed steps)
    match_ms = sum(float(r[3][2]) for r in recs)
    upd_ms = sum(float(r[3][0]) for r in recs)
    match_bytes = sum(r[4]["match_bytes"] for r in recs)
    upd_bytes = sum(r[4]["update_bytes"] for r in recs)
    peak, peak_kind = _peaks()
    if match_ms >= upd_ms:
        kname, kbytes, kms = "k_dfs_count (matching)", match_bytes, match_ms
    else:
        kname, kbytes, kms = "k_merge_runs (index update)", upd_bytes, upd_ms
    traffic, traffic_src = _profiled_traffic(kname.split()[0])
    achieved = (kbytes / 1e9) / (kms / 1e3) if kms > 0 else 0.0
    upd_achieved = (upd_bytes / 1e9) / (upd_ms / 1e3) if upd_ms > 0 else 0.0
    lat = sorted(step_ms)

    def pct(p):
        return lat[min(len(lat) - 1, int(round(p / 100.0 * (len(lat) - 1))))]

    line = {
        "metric": "edge updates/sec (and incremental matches/sec, p50/p99 batch latency) on 1 B200",
        "value": edges / (total_ms / 1e3) if total_ms > 0 else 0.0,
        "unit": "edge updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / max(1, len(recs)),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32/u64 integer", "data": "synthetic (seeded R-MAT stand-in for the public graphs)",
        "config": {"workload": "R-MAT 1,000,000 vertices / 10,000,000 edges, 16 labels Zipf(1.2), "
                               "1,000,000 insertions in batches of 100,000, 9-vertex dense pattern",
                   "batch_edges": spec.batch_edges, "batches_in_stream": nb,
                   "query_vertices": len(ql), "query_edges": len(qe),
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"{world} GPU(s): index replicated, seeds sharded"},
        "matches_per_s": matches / (total_ms / 1e3) if total_ms > 0 else 0.0,
        "matches_per_batch": matches / max(1, len(recs)),
        "latency_ms": {"p50": pct(50), "p99": pct(99), "max": lat[-1]},
        "phase_ms_per_step": {"index_update": upd_ms / len(recs),
                              "delta_lists": sum(float(r[3][1]) for r in recs) / len(recs),
                              "matching": match_ms / len(recs)},
        "work_per_step": {k: sum(r[4][k] for r in recs) / len(recs)
                          for k in ("seeds", "chunks", "tested", "tails", "stolen_tasks", "touched_runs")},
        "e2e": {"value": e2e_edges / (e2e_ms / 1e3) if e2e_ms > 0 else 0.0, "unit": "edge updates/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 8 * (4 + 16 + 8)},
        "gpu_launches": launches,
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak if peak else None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": kbytes / len(recs), "traffic": traffic,
                     "traffic_source": traffic_src,
                     "index_update_achieved_gbs": upd_achieved},
        "clocks": clk.summary(),
        "stage1_setup_s": round(s1_s, 2),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import bind

        if bind.have_ref():
            log("cpu baseline: reference CPU path on batch 0")
            line["cpu_baseline"] = reference_sample(paths, spec, args.cpu_budget_s, batches)
        else:
            line["cpu_baseline"] = {"unavailable": "oracle/_ref/libcgbref.so was not built (no reference tree)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    state["eng"].close()
    dist.finish()


def reference_sample(paths, spec, budget_s: float, batches=None) -> dict:
    """The reference's own CPU path (oracle/_ref: CaLiG + staging + CPUIndexMirror +
    cpu_dfs) on batch 0 of the same stream with all host threads.  Stage 1,
    staging and the index mirror update run fully; the count (the reference
    enumerates every embedding, mask-free seeding) runs for budget_s in a
    supervised child process and is extrapolated by rows counted / rows total.
    When not one row finishes in the budget, the count time is bounded below by
    budget_s x rows_total and the value is an upper bound."""
    from oracle import bind

    threads = os.cpu_count() or 1
    r = bind.supervised_reference_batch(paths["query"], paths["data"], paths["update"], spec.cli_batch_size,
                                        threads, budget_s)
    fixed_ms = r["s1_ms"] + r["staging_ms"] + r["mirror_ms"]
    if r["finished"]:
        count_ms, kind = r["count_ms"], "measured"
    elif r["rows_done"] > 0:
        count_ms, kind = r["count_ms"] * r["rows_total"] / r["rows_done"], "extrapolated"
    else:
        count_ms, kind = r["count_ms"] * max(1, r["rows_total"]), "lower bound (no row finished)"
    batch_ms = fixed_ms + count_ms
    value = spec.batch_edges / (batch_ms / 1e3) if batch_ms > 0 else 0.0
    return {"value": value, "unit": "edge updates/s", "cores": threads, "kind": "reference",
            "sample": (f"batch 0 of the stream: Stage 1 {r['s1_ms']:.0f} ms + staging {r['staging_ms']:.0f} ms + "
                       f"index mirror {r['mirror_ms']:.0f} ms measured; mask-free cpu_dfs count: "
                       f"{r['rows_done']} of {r['rows_total']} seed rows in {r['count_ms']/1e3:.1f} s, "
                       f"count time {kind}: {count_ms/1e3:.3g} s"
                       + ("; value is an upper bound" if kind.startswith("lower") else "")),
            "stage1_ms": r["s1_ms"], "count_time_kind": kind, "wall_s": round(r["wall_s"], 1)}


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cgbdsm_b200.workloads import SPECS, materialize

    spec = SPECS[WORKLOAD]
    paths = materialize(spec, os.environ.get("CGB_BENCH_DIR", "/tmp/cgb_bench_r0"))
    from oracle import bind

    if not bind.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcgbref.so was not built"}))
        return
    vals = []
    cb = None
    per_step_budget = max(2.0, min(args.cpu_budget_s, 150.0 / max(1, args.steps + args.warmup)))
    for i in range(args.warmup + args.steps):
        cb = reference_sample(paths, spec, per_step_budget)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals) if vals else 0.0
    cb["value"] = v
    print(json.dumps({
        "impl": "reference",
        "metric": "edge updates/sec (and incremental matches/sec, p50/p99 batch latency) on 1 B200",
        "value": v, "unit": "edge updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": (spec.batch_edges / v * 1e3) if v else None, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32/u64 integer", "data": "synthetic (seeded R-MAT)",
        "config": {"workload": "R-MAT 1,000,000 vertices / 10,000,000 edges, 16 labels Zipf(1.2), "
                               "1,000,000 insertions in batches of 100,000, 9-vertex dense pattern"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "edge updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=7)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--budget-ms", type=int, default=120000, help="matching time budget per batch")
    ap.add_argument("--cpu-budget-s", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="profiling run: 1 warm-up + 1 step, no e2e leg, no CPU baseline (not a benchmark)")
    args = ap.parse_args()
    if args.quick:
        args.steps, args.warmup, args.no_cpu_baseline = 1, 1, True
    elif args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
