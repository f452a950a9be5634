"""Golden shard counts for the R-MAT 1M/10M benchmark pattern (and others),
from the oracle's independent counted-tail restatement (oracle/oracle.c,
ORC_TAIL mode, itself pinned to the reference's CPU path by
tests/test_oracle_pin.py).

The benchmark stream's counts (~10^16 matches per batch) are far beyond what
an enumerating CPU count can reach, so the check is made on shards of the seed
groups: the oracle counts only the seeds whose group key (query edge ei, data
vertex at the plan's first query vertex) hashes to a given shard, exactly as
the engine's cgb_config.shard_index / num_shards select them.  The keys come
from the product's Stage-1 producer (its key multisets equal the reference's
on this stream, tests/test_producer.py).  Writes tests/golden/shards_<name>.json:

    python tests/golden/make_shard_golden.py c2 256 0,1,2,3

(one process per shard; several minutes of CPU per shard at 256 shards).
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def plan_anchor(qv: int, qedges) -> list[int]:
    """The engine's plan anchor of each query edge (reference edge order): the
    edge's first endpoint, unless that one is a pendant and the other is not."""
    deg = [0] * qv
    for a, b in qedges:
        deg[a] += 1
        deg[b] += 1
    edges = sorted((min(a, b), max(a, b)) for a, b in qedges)
    return [v if (deg[u] == 1 and deg[v] > 1) else u for u, v in edges]


def shard_counts(name: str, batches: int, num_shards: int, shard: int, workdir: str) -> dict:
    from cgbdsm_b200 import Producer
    from cgbdsm_b200.workloads import SPECS, materialize, read_query
    from oracle import bind

    spec = SPECS[name]
    p = materialize(spec, workdir)
    ql, qe = read_query(p["query"])
    prod = Producer(p["query"], p["data"], p["update"], spec.cli_batch_size)
    init, dv = prod.initial()
    o = bind.Oracle(len(ql), qe)
    o.set_shard(shard, num_shards, plan_anchor(len(ql), qe))
    o.build(init, dv)
    out = []
    for b in range(batches):
        r = prod.next()
        t0 = time.time()
        c = o.batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"], bind.TAIL)
        out.append({"batch": b, "count": c, "edge_counts": [int(x) for x in o.edge_counts()],
                    "cpu_s": round(time.time() - t0, 1)})
    prod.close()
    return {"shard": shard, "batches": out}


def _job(args):
    return shard_counts(*args)


def main() -> None:
    from cgbdsm_b200.workloads import SPECS, read_query, materialize

    name, num_shards = sys.argv[1], int(sys.argv[2])
    shards = [int(x) for x in sys.argv[3].split(",")]
    batches = int(sys.argv[4]) if len(sys.argv) > 4 else 1
    workdir = os.environ.get("CGB_GOLDEN_DIR", "/tmp/cgb_golden")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ql, qe = read_query(p["query"])
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(shards)) as pool:
        res = pool.map(_job, [(name, batches, num_shards, s, workdir) for s in shards])
    rec = {"workload": name, "spec": repr(spec), "num_shards": num_shards,
           "anchors": plan_anchor(len(ql), qe), "mode": "oracle counted tail (ORC_TAIL)", "shards": res}
    with open(os.path.join(HERE, f"shards_{name}.json"), "w") as f:
        json.dump(rec, f, indent=1)
        f.write("\n")
    print(json.dumps(rec)[:400])


if __name__ == "__main__":
    main()
