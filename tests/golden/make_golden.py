"""Generates the golden fixtures in this directory from the reference's own CPU
path (oracle/_ref/libcgbref.so, built from the reference sources by
oracle/Makefile).  Run in a container that holds the reference tree:

    CGB_REFERENCE_TREE=/root/reference python tests/golden/make_golden.py

For each workload it records what the reference computes on the seeded
synthetic input (cgbdsm_b200/workloads.py):

  * sha256 of the three input files (pins the generator),
  * per batch: compressed-vertex count, edge_ok flags, match count, and the
    ins / del / delta key multisets as (length, sha256) in ORIGINAL vertex ids
    (ins as a set: the reference deduplicates it downstream,
    index/calig_helper_gamma.cu:254-256),
  * the initial and final index contents, (length, sha256) in original ids.

t_tiny is stored in full as well (inputs, keys in the reference's own
compressed ids, new->old mapping, final index) so the restatement can be
replayed from the fixture alone.  <name>_csr.json holds the same digests for
the reference's binary CSR input path (labels drawn from rand(), hash-selected
update stream) on the full graph of <name>.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cgbdsm_b200.workloads import SPECS, materialize, write_binary_csr  # noqa: E402
from oracle import bind  # noqa: E402

FULL = ["t_tiny"]
HASHED = ["t_tiny", "t_er5", "t_er_tree", "t_er_sparse", "t_rmat", "c1", "c1_q25"]
# binary CSR inputs (calig.cpp:218-323): workload -> number of vertex classes
BINARY = {"t_er5": 4, "t_rmat": 10}


def to_original(keys: np.ndarray, new2old: np.ndarray) -> np.ndarray:
    n2o = new2old.astype(np.uint64)
    d = keys >> np.uint64(59)
    u = (keys >> np.uint64(32)) & np.uint64(0x7FFFFFF)
    v = keys & np.uint64(0xFFFFFFFF)
    return np.sort((d << np.uint64(59)) | (n2o[u] << np.uint64(32)) | n2o[v])


def digest(keys: np.ndarray) -> list:
    a = np.ascontiguousarray(np.sort(keys).astype("<u8"))
    return [int(a.size), hashlib.sha256(a.tobytes()).hexdigest()]


def file_digest(path: str) -> str:
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def make(name: str, workdir: str) -> None:
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    rec = {
        "workload": name,
        "spec": repr(spec),
        "inputs": {k: file_digest(v) for k, v in p.items()},
        "num_batches": ref.num_batches,
        "dv_initial": ref.dv_count,
        "initial_index": digest(to_original(ref.init_keys(), ref.new2old())),
        "batches": [],
    }
    full = {"init": ref.init_keys(), "dv0": np.uint32(ref.dv_count)}
    for f in ("query", "data", "update"):
        full["file_" + f] = np.frombuffer(open(p[f], "rb").read(), dtype=np.uint8)
    while True:
        b = ref.step()
        if b < 0:
            break
        r = ref.last()
        n2o = ref.new2old()
        rec["batches"].append({
            "dv": int(r["dv"]),
            "edge_ok": [int(x) for x in r["edge_ok"]],
            "count": int(r["count"]),
            "ins": digest(np.unique(to_original(r["ins"], n2o))),
            "del": digest(to_original(r["del"], n2o)),
            "delta": digest(to_original(r["delta"], n2o)),
        })
        for k in ("ins", "del", "delta"):
            full[f"b{b}_{k}"] = r[k]
        full[f"b{b}_edge_ok"] = r["edge_ok"]
        full[f"b{b}_meta"] = np.array([r["dv"], r["count"]], dtype=np.uint64)
    final = ref.dump_main_original_ids()
    rec["final_index"] = digest(final)
    full["final_original"] = final
    full["new2old"] = ref.new2old()
    ref.close()
    with open(os.path.join(HERE, f"{name}.json"), "w") as f:
        json.dump(rec, f, indent=1)
        f.write("\n")
    if name in FULL:
        np.savez_compressed(os.path.join(HERE, f"{name}_full.npz"), **full)
    print(name, rec["num_batches"], "batches, counts", [b["count"] for b in rec["batches"]])


def make_binary(name: str, nvcls: int, workdir: str) -> None:
    """The reference reads the CSR prefix and draws labels from rand(), so it
    runs in a fresh process (oracle/refdigest.py)."""
    import subprocess

    spec = SPECS[name]
    p = write_binary_csr(spec, workdir, nvcls)
    r = subprocess.run([sys.executable, "-m", "oracle.refdigest", p["query"], p["data"], "-",
                        str(spec.cli_batch_size)], capture_output=True, text=True, check=True, cwd=ROOT)
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    rec = {"workload": name, "spec": repr(spec), "nvcls": nvcls,
           "inputs": {s: file_digest(p["data"] + s) for s in (".meta.txt", ".vertex.bin", ".edge.bin")}, **rec}
    with open(os.path.join(HERE, f"{name}_csr.json"), "w") as f:
        json.dump(rec, f, indent=1)
        f.write("\n")
    print(name, "binary CSR,", rec["num_batches"], "batches, counts", [b["count"] for b in rec["batches"]])


def main() -> None:
    bind.build(ref=True)
    if not bind.have_ref():
        raise SystemExit("oracle/_ref/libcgbref.so could not be built (reference tree absent)")
    only = set(sys.argv[1:])  # optional: regenerate only these fixtures
    with tempfile.TemporaryDirectory() as d:
        for name in HASHED:
            if not only or name in only:
                make(name, d)
        for name, nvcls in BINARY.items():
            if not only or f"{name}_csr" in only:
                make_binary(name, nvcls, d)


if __name__ == "__main__":
    main()
