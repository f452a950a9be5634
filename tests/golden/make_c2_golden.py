"""Golden counts of the reference's own CPU path (oracle/_ref: CaLiG +
staging + CPUIndexMirror + cpu_dfs) on the full R-MAT 1M/10M stream for
patterns of the stored 64-query set whose counts an enumerating CPU count
can reach (cgbdsm_b200/data/queries_c2.json; the benchmark's 9-vertex dense
family has none under 10^11 matches per batch).  Run where the reference
tree is present:

    CGB_REFERENCE_TREE=/root/reference python tests/golden/make_c2_golden.py

Writes tests/golden/c2_patterns.json: per pattern its labels, edges and the
reference's count for each batch it ran (all 10 batches for the fast ones).
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cgbdsm_b200.workloads import SPECS, materialize  # noqa: E402
from oracle import bind  # noqa: E402

# (index in queries_c2.json, batches to run)
PATTERNS = [(33, 10), (18, 10), (12, 1)]


def main() -> None:
    bind.build(ref=True)
    if not bind.have_ref():
        raise SystemExit("oracle/_ref/libcgbref.so could not be built (reference tree absent)")
    qs = json.load(open(os.path.join(ROOT, "cgbdsm_b200", "data", "queries_c2.json")))["queries"]
    spec = SPECS["c2"]
    workdir = os.environ.get("CGB_GOLDEN_DIR", "/tmp/cgb_golden")
    p = materialize(spec, workdir)
    out = {"workload": "c2", "spec": repr(spec), "patterns": []}
    for k, nb in PATTERNS:
        q = qs[k]
        qp = os.path.join(workdir, "c2", f"golden_q{k}.graph")
        with open(qp, "w") as f:
            for i, lb in enumerate(q["labels"]):
                f.write(f"v {i} {lb}\n")
            for a, b in q["edges"]:
                f.write(f"e {a} {b} 0\n")
        ref = bind.RefPipeline(qp, p["data"], p["update"], spec.cli_batch_size, threads=os.cpu_count() or 1)
        counts, secs = [], []
        for _ in range(nb):
            t0 = time.time()
            ref.step()
            counts.append(int(ref.last()["count"]))
            secs.append(round(time.time() - t0, 1))
        ref.close()
        out["patterns"].append({"index": k, "shape": q["shape"], "labels": q["labels"], "edges": q["edges"],
                                "reference_counts": counts, "reference_seconds": secs})
        print(k, counts, secs, flush=True)
    with open(os.path.join(HERE, "c2_patterns.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
