"""Digests of the reference CPU path's per-batch outputs, run in a process of
its own.  TEST INFRASTRUCTURE ONLY (tests/ and tests/golden/make_golden.py).

The reference's binary reader draws vertex labels from the C library's rand()
(calig.cpp:269), so it must run in a fresh process where nothing else has
drawn from that sequence:

    python -m oracle.refdigest <query> <data> <update> <batch_size_ints>

prints one JSON object: initial-index digest, per batch (vertex count,
edge_ok, count, ins / del / delta digests in original ids), final-index
digest.  A digest is [length, sha256 of the sorted little-endian u64 keys].
"""
from __future__ import annotations

import hashlib
import json
import sys

import numpy as np


def to_original(keys: np.ndarray, new2old: np.ndarray) -> np.ndarray:
    n2o = new2old.astype(np.uint64)
    d = keys >> np.uint64(59)
    u = (keys >> np.uint64(32)) & np.uint64(0x7FFFFFF)
    v = keys & np.uint64(0xFFFFFFFF)
    return np.sort((d << np.uint64(59)) | (n2o[u] << np.uint64(32)) | n2o[v])


def digest(keys: np.ndarray) -> list:
    a = np.ascontiguousarray(np.sort(keys).astype("<u8"))
    return [int(a.size), hashlib.sha256(a.tobytes()).hexdigest()]


def run(query: str, data: str, update: str, batch_size_ints: int) -> dict:
    from oracle import bind

    ref = bind.RefPipeline(query, data, update, batch_size_ints)
    out = {"num_batches": ref.num_batches, "dv_initial": ref.dv_count,
           "initial_index": digest(to_original(ref.init_keys(), ref.new2old())), "batches": []}
    while ref.step() >= 0:
        r = ref.last()
        n2o = ref.new2old()
        out["batches"].append({
            "dv": int(r["dv"]), "edge_ok": [int(x) for x in r["edge_ok"]], "count": int(r["count"]),
            "ins": digest(np.unique(to_original(r["ins"], n2o))),
            "del": digest(to_original(r["del"], n2o)),
            "delta": digest(to_original(r["delta"], n2o)),
        })
    out["final_index"] = digest(ref.dump_main_original_ids())
    ref.close()
    return out


if __name__ == "__main__":
    q, d, u, b = sys.argv[1], sys.argv[2], sys.argv[3], int(sys.argv[4])
    print(json.dumps(run(q, d, u, b)))
