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
    python -m cgbdsm_b200.queryset c3_tree 64   # R-MAT 4M/34M graph (serving mix)
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


if __name__ == "__main__":
    name, n = sys.argv[1], int(sys.argv[2])
    out = select(name, n)
    os.makedirs(DATA, exist_ok=True)
    dest = sys.argv[3] if len(sys.argv) > 3 else path(name)
    with open(dest, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(f"{len(out['queries'])} queries, {len(out['skipped'])} skipped -> {dest}")
