"""Query sets of the multi-query and serving workloads.

Mix: query sizes drawn uniformly from 4..12 vertices, shapes split between
tree, sparse and dense random-walk patterns (21 / 21 / 22 of 64), sampled
from the workload's final graph (cgbdsm_b200/workloads.GraphData.query).
Selection rule: a pattern whose first batch yields more than 10^11 positive
matches, or whose first batch does not finish within the per-query matching
budget on a B200, is replaced by the next query seed of the same shape and
size; after ATTEMPTS seeds at one size the size is lowered by one (R-MAT
graphs put a hub in almost every 10-12 vertex sample, and those patterns
have ~10^18 embeddings per batch); skipped seeds and the drawn and used
sizes are recorded.  The rule needs a GPU, so the chosen set is computed once
and stored (cgbdsm_b200/data/queries_<name>.json):

    python -m cgbdsm_b200.queryset c2 64        # R-MAT 1M/10M graph, 64 queries
    python -m cgbdsm_b200.queryset c3_tree 16   # R-MAT 4M/34M graph (serving mix)

Two more reports on a workload's own pattern family (shape and size of its
spec, query seeds varied), through the plain single-query pipeline (CaLiG
producer + engine), first batch:

    python -m cgbdsm_b200.queryset sweep c2 24 43      # ms or budget hit per seed
    python -m cgbdsm_b200.queryset find c2 42 400 3    # first 3 seeds with <= 10^11 matches
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")
MAX_MATCHES = 10**11       # per query and batch (the reseed rule)
BUDGET_MS = 500            # matching budget of one query alone on the first batch
ATTEMPTS = 4               # seeds tried per size before the size is lowered
SHAPES = {0: "dense", 1: "sparse", 2: "tree"}


def mix(n: int, seed: int = 44) -> list[tuple[int, int]]:
    """(shape, size) of n queries: sizes U{4..12}; 21/21/22 tree/sparse/dense per 64."""
    rng = np.random.default_rng(seed)
    shapes = [2] * (n * 21 // 64) + [1] * (n * 21 // 64)
    shapes += [0] * (n - len(shapes))
    rng.shuffle(shapes)
    sizes = rng.integers(4, 13, n)
    return [(int(s), int(z)) for s, z in zip(shapes, sizes)]


def path(name: str) -> str:
    return os.path.join(DATA, f"queries_{name}.json")


def load(name: str) -> list[dict]:
    """The stored query set: [{"labels", "edges", "shape", "size", "seed"}, ...]."""
    with open(path(name)) as f:
        return json.load(f)["queries"]


def select(workload: str, n: int, first_seed: int = 1000) -> dict:
    from .engine import MQ_FLAG_NO_AUTOTUNE, CgbError, MultiQuery
    from .workloads import SPECS, GraphData

    spec = SPECS[workload]
    g = GraphData(spec)
    first = g.batches()[0]
    chosen, skipped = [], []
    seed = first_seed
    # one engine: each candidate alone matches the first batch, which is then
    # deleted again (with no query registered) to restore the initial graph
    m = MultiQuery(dfs_budget_ms=BUDGET_MS, flags=MQ_FLAG_NO_AUTOTUNE)
    m.load_graph(g.labels, g.initial)
    for shape, drawn in mix(n):
        size, tries = drawn, 0
        while True:
            if tries == ATTEMPTS and size > 4:
                size, tries = size - 1, 0
            seed += 1
            tries += 1
            q = g.query(shape, size, seed, 32)
            if q is None:
                skipped.append({"shape": SHAPES[shape], "size": size, "seed": seed, "why": "no pattern"})
                continue
            ql, qe = q
            qid = m.register(len(ql), qe, ql)
            t0 = time.time()
            ok = True
            try:
                pos, _ = m.apply_batch(ins=first)
                cnt, why = int(pos[qid]), None
                if cnt > MAX_MATCHES:
                    why = f"{cnt} matches on the first batch"
            except CgbError as e:
                cnt, why, ok = None, f"matching budget ({e.status})", False
            ms = float(m.timings()[2]) if ok else (time.time() - t0) * 1e3
            m.unregister(qid)
            if ok:
                m.apply_batch(dele=first)
            rec = {"shape": SHAPES[shape], "size": size, "seed": seed, "qv": len(ql), "qe": len(qe)}
            if why:
                skipped.append({**rec, "why": why})
                print(f"skip {rec}: {why}", flush=True)
                continue
            chosen.append({**rec, "size_drawn": drawn, "labels": ql, "edges": [list(e) for e in qe],
                           "first_batch_count": cnt, "first_batch_ms_alone": round(ms, 3)})
            print(f"keep {rec} (drawn {drawn}): {cnt} matches, {ms:.1f} ms", flush=True)
            break
    m.close()
    return {"workload": workload, "spec": repr(spec), "rule": f"> {MAX_MATCHES} matches or > {BUDGET_MS} ms on "
            "the first batch alone: next seed", "queries": chosen, "skipped": skipped}


def plain_first_batch(workload: str, g, seed: int, budget_ms: int, workdir: str) -> dict:
    """The spec's pattern family with query seed `seed` through the plain
    pipeline: edges, first-batch count and matching time, or the budget hit.
    g: the workload's GraphData (the same sampler materialize() uses)."""
    from .engine import CgbError, Engine, Producer
    from .workloads import SPECS, materialize

    spec = SPECS[workload]
    p = materialize(spec, workdir)
    q = g.query(spec.qshape, spec.qsize, seed, spec.max_qedges)
    if q is None:
        return {"seed": seed, "no_pattern": True}
    ql, qe = q
    qpath = os.path.join(os.path.dirname(p["query"]), f"query_s{seed}.graph")
    with open(qpath, "w") as f:
        for i, lb in enumerate(ql):
            f.write(f"v {i} {lb}\n")
        for a, b in qe:
            f.write(f"e {a} {b} 0\n")
    prod = Producer(qpath, p["data"], p["update"], spec.cli_batch_size)
    init, dv = prod.initial()
    r = prod.next()
    prod.close()
    e = Engine(dfs_budget_ms=budget_ms)
    e.load_query(len(ql), qe, ql)
    e.build_index(init, dv)
    out = {"seed": seed, "qv": len(ql), "qe": len(qe), "query_file": qpath}
    try:
        out["count"] = e.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
        out["match_ms"] = round(float(e.timings()[2]), 2)
    except CgbError as err:
        out["budget_hit"] = f"> {budget_ms} ms ({err.status})"
    e.close()
    return out


def _report(argv) -> None:
    from .workloads import SPECS, GraphData

    workdir = os.environ.get("CGB_BENCH_DIR", "/tmp/cgb_queryset")
    cmd, workload, lo, hi = argv[0], argv[1], int(argv[2]), int(argv[3])
    g = GraphData(SPECS[workload])
    if cmd == "sweep":
        for seed in range(lo, hi + 1):
            print(json.dumps(plain_first_batch(workload, g, seed, 3000, workdir)), flush=True)
        return
    want = int(argv[4]) if len(argv) > 4 else 1
    found = 0
    for seed in range(lo, hi + 1):
        r = plain_first_batch(workload, g, seed, BUDGET_MS, workdir)
        ok = "count" in r and r["count"] <= MAX_MATCHES
        print(json.dumps({**r, "kept": ok}), flush=True)
        found += ok
        if found >= want:
            break


if __name__ == "__main__":
    if sys.argv[1] in ("sweep", "find"):
        _report(sys.argv[1:])
        sys.exit(0)
    name, n = sys.argv[1], int(sys.argv[2])
    out = select(name, n)
    os.makedirs(DATA, exist_ok=True)
    dest = sys.argv[3] if len(sys.argv) > 3 else path(name)
    with open(dest, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"{len(out['queries'])} queries, {len(out['skipped'])} skipped -> {dest}")
