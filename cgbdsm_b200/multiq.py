"""Multi-query workload: 64 registered queries on the R-MAT 1M/10M stream.

The multi-query engine (cgb_mq_*) keeps one data-graph index on the device
and matches all 64 queries per batch in one persistent launch; the plain
pipeline runs each query through its own CaLiG producer (Stage 1, host) and
single-query engine (one launch per query and batch), as the reference runs
one query per process (main_calig.cpp:203-384).  Both process the same
batches, and every query's count is compared between them, batch by batch.

Timing: the multi-query engine takes batch 0 as warm-up (the autotuner runs
there, untimed) and is timed on batches 1-9: device time per batch (CUDA
events) for the value, and the host-buffer C-ABI call (H2D of the edge
pairs, matching, D2H of the counts) for e2e.  The plain pipeline is timed on
batches 1-3 (its Stage-1 index build per query takes ~1.5 s, 64 times):
  gpu    sum over queries of the engine's device time per batch
  e2e    sum over queries of max(Stage 1, Stage 2) per batch: each query's
         two-stage pipeline overlapped, queries one after another
Patterns with more than 16 edges have no CaLiG key encoding (5-bit directed
edge index); for them the plain pipeline is the multi-query engine holding
that query alone (one launch per query), without a Stage 1.
"""
from __future__ import annotations

import os
import time

import numpy as np

PLAIN_BATCHES = (1, 2, 3)


def _write_query(path: str, q: dict) -> None:
    with open(path, "w") as f:
        for i, lb in enumerate(q["labels"]):
            f.write(f"v {i} {lb}\n")
        for a, b in q["edges"]:
            f.write(f"e {a} {b} 0\n")


def bench(args, local: int, log) -> dict:
    import torch

    from . import queryset
    from .engine import MQ_FLAG_NO_AUTOTUNE, Engine, MultiQuery, Producer
    from .workloads import SPECS, GraphData, materialize

    spec = SPECS["c2"]
    qs = queryset.load("c2")
    g = GraphData(spec)
    batches = g.batches()
    dev = f"cuda:{local}"
    budget = args.budget_ms

    def engine(flags=0):
        m = MultiQuery(device=local, dfs_budget_ms=budget, flags=flags)
        m.load_graph(g.labels, g.initial)
        ids = [m.register(q["qv"], [tuple(e) for e in q["edges"]], q["labels"]) for q in qs]
        return m, ids

    # ---- multi-query engine, device-resident edge pairs
    log(f"c4: multi-query engine, {len(qs)} queries")
    m, ids = engine()
    dpairs = [torch.from_numpy(b.astype(np.int32).reshape(-1)).to(dev) for b in batches]
    torch.cuda.synchronize()
    counts, ms, lat, launches, t_phase, merge_bytes = {}, [], [], 0, np.zeros(3), 0
    for b in range(len(batches)):
        l0 = m.kernel_launches()
        pos, _ = m.apply_batch_device(dpairs[b].data_ptr(), len(batches[b]))
        t = m.timings()
        counts[b] = [int(pos[i]) for i in ids]
        if b >= 1:
            ms.append(float(t[3]))
            t_phase += np.array([float(x) for x in t[:3]])
            launches += m.kernel_launches() - l0
            merge_bytes += m.stats()["update_bytes"]
        log(f"c4 batch {b}: {float(t[3]):.1f} ms (merge {float(t[0]):.2f}, delta {float(t[1]):.2f}, match "
            f"{float(t[2]):.1f})")
    variants = [m.query_info(i) for i in ids]
    sched = m.schedule()
    m.close()
    timed = list(range(1, len(batches)))
    edges = sum(len(batches[b]) for b in timed)
    dev_ms = sum(ms)

    # ---- the same through the host-buffer C-ABI call (e2e)
    m, ids = engine()
    m.apply_batch(ins=batches[0])  # warm-up and autotune
    e2e_ms = []
    for b in timed:
        t0 = time.perf_counter()
        pos, _ = m.apply_batch(ins=batches[b])
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        assert [int(pos[i]) for i in ids] == counts[b]
    m.close()

    # ---- plain pipeline, one query at a time
    log("c4: plain pipeline (CaLiG producer + single-query engine per query)")
    p = materialize(spec, os.environ.get("CGB_BENCH_DIR", "/tmp/cgb_bench"))
    qdir = os.path.join(os.path.dirname(p["query"]), "c4_queries")
    os.makedirs(qdir, exist_ok=True)
    plain_gpu = {b: 0.0 for b in PLAIN_BATCHES}
    plain_e2e = {b: 0.0 for b in PLAIN_BATCHES}
    mismatches, keyed, s1_init = [], 0, 0.0
    for k, q in enumerate(qs):
        if q["qe"] <= 16:
            keyed += 1
            qp = os.path.join(qdir, f"q{k}.graph")
            _write_query(qp, q)
            t0 = time.perf_counter()
            prod = Producer(qp, p["data"], p["update"], spec.cli_batch_size)
            init, dv = prod.initial()
            s1_init += time.perf_counter() - t0
            e = Engine(device=local, dfs_budget_ms=budget)
            e.load_query(q["qv"], [tuple(x) for x in q["edges"]], q["labels"])
            e.build_index(init, dv)
            for b in range(max(PLAIN_BATCHES) + 1):
                t0 = time.perf_counter()
                r = prod.next()
                s1 = (time.perf_counter() - t0) * 1e3
                c = e.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
                if c != counts[b][k]:
                    mismatches.append({"query": k, "batch": b, "plain": c, "multi": counts[b][k]})
                if b in PLAIN_BATCHES:
                    s2 = float(e.timings()[3])
                    plain_gpu[b] += s2
                    plain_e2e[b] += max(s1, s2)
            e.close()
            prod.close()
        else:
            one = MultiQuery(device=local, dfs_budget_ms=budget, flags=MQ_FLAG_NO_AUTOTUNE)
            one.load_graph(g.labels, g.initial)
            qid = one.register(q["qv"], [tuple(x) for x in q["edges"]], q["labels"])
            for b in range(max(PLAIN_BATCHES) + 1):
                pos, _ = one.apply_batch(ins=batches[b])
                if int(pos[qid]) != counts[b][k]:
                    mismatches.append({"query": k, "batch": b, "plain": int(pos[qid]), "multi": counts[b][k]})
                if b in PLAIN_BATCHES:
                    s2 = float(one.timings()[3])
                    plain_gpu[b] += s2
                    plain_e2e[b] += s2
            one.close()
    pb_edges = sum(len(batches[b]) for b in PLAIN_BATCHES)
    mq_pb_ms = sum(ms[b - 1] for b in PLAIN_BATCHES)
    mq_pb_e2e = sum(e2e_ms[b - 1] for b in PLAIN_BATCHES)
    plain_gpu_ms, plain_e2e_ms = sum(plain_gpu.values()), sum(plain_e2e.values())
    shapes = {}
    for q in qs:
        shapes[q["shape"]] = shapes.get(q["shape"], 0) + 1
    return {
        "metric": "edge updates/sec with 64 registered queries (each batch matched for every query)",
        "value": edges / (dev_ms / 1e3), "unit": "edge updates/s",
        "config": {"workload": "R-MAT 1,000,000 / 10,000,000, 16 labels Zipf(1.2), batches of 100,000; "
                               f"{len(qs)} queries (sizes {min(q['qv'] for q in qs)}-{max(q['qv'] for q in qs)}, "
                               f"{shapes}), cgbdsm_b200/data/queries_c2.json",
                   "timed_batches": timed, "warmup_batches": [0]},
        "ms_per_batch": dev_ms / len(ms),
        "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99)), "max": max(ms)},
        "phase_ms_per_batch": {"index_merge": t_phase[0] / len(ms), "delta": t_phase[1] / len(ms),
                               "matching": t_phase[2] / len(ms)},
        "index_merge_achieved_gbs": (merge_bytes / 1e9) / (t_phase[0] / 1e3) if t_phase[0] > 0 else None,
        "matches_per_s": sum(sum(counts[b]) for b in timed) / (dev_ms / 1e3),
        "e2e": {"value": edges / (sum(e2e_ms) / 1e3), "unit": "edge updates/s",
                "h2d_bytes_per_step": int(8 * np.mean([len(batches[b]) for b in timed])),
                "d2h_bytes_per_step": 8 * 2 * 256},
        "gpu_launches": launches,
        "autotune": {"blocks_per_sm": sched[0], "steal": sched[1],
                     "variants": {str(v): sum(1 for x in variants if x[0] == v) for v in sorted({x[0] for x in variants})}},
        "plain_pipeline": {
            "batches": list(PLAIN_BATCHES), "queries_with_calig_keys": keyed,
            "gpu_value": pb_edges / (plain_gpu_ms / 1e3), "e2e_value": pb_edges / (plain_e2e_ms / 1e3),
            "gpu_ms_per_batch": plain_gpu_ms / len(PLAIN_BATCHES), "e2e_ms_per_batch": plain_e2e_ms / len(PLAIN_BATCHES),
            "stage1_index_build_s_total": round(s1_init, 1),
            "speedup_gpu": plain_gpu_ms / mq_pb_ms, "speedup_e2e": plain_e2e_ms / mq_pb_e2e,
        },
        "counts_equal_plain": not mismatches, "count_mismatches": mismatches[:10],
    }


def profile_run(batches: int = 2, queries: int = 64) -> None:
    """The multi-query engine alone on the R-MAT 1M/10M stream with the stored
    query set (first `queries`), `batches` batches: the command profiles use
    (python -m cgbdsm_b200.multiq [batches] [queries])."""
    from . import queryset
    from .engine import MultiQuery
    from .workloads import SPECS, GraphData

    g = GraphData(SPECS["c2"])
    qs = queryset.load("c2")[:queries]
    m = MultiQuery(dfs_budget_ms=120000)
    m.load_graph(g.labels, g.initial)
    ids = [m.register(q["qv"], [tuple(e) for e in q["edges"]], q["labels"]) for q in qs]
    for b, batch in enumerate(g.batches()[:batches]):
        pos, _ = m.apply_batch(ins=batch)
        t = m.timings()
        st = m.stats()
        print(f"batch {b}: {float(t[3]):.1f} ms (merge {float(t[0]):.2f} ms, {st['update_bytes']} B; delta "
              f"{float(t[1]):.2f} ms; match {float(t[2]):.1f} ms), total count {int(sum(int(pos[i]) for i in ids))}",
              flush=True)
    m.close()


if __name__ == "__main__":
    import sys

    profile_run(*(int(x) for x in sys.argv[1:3]))
