"""ctypes bindings of the oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's reference / cpu_baseline legs as the checker; the product never
imports it.

  RefPipeline  oracle/_ref/libcgbref.so: the reference's own CPU path
               (CaLiG + host staging + CPUIndexMirror + cpu_dfs)
  Oracle       oracle/liboracle.so: the plain-C restatement (oracle.c)
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libcgbref.so")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
# The reference source tree, when this machine has one (only `build` reads it).
REF_TREE = os.environ.get("CGB_REFERENCE_TREE", "")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32, _u64, _vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p

GLOBAL, PER_EDGE, TAIL = 0, 1, 2


def build(ref: bool = True, ref_tree: Optional[str] = None) -> None:
    """Builds liboracle.so, and libcgbref.so when a reference source tree is
    given (ref_tree, else $CGB_REFERENCE_TREE) and present on this machine."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    tree = ref_tree or REF_TREE
    if ref and tree and os.path.isdir(tree):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={tree}"], check=True)


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def _as_np(p, n) -> np.ndarray:
    if n == 0:
        return np.zeros(0, dtype=np.uint64)
    return np.ctypeslib.as_array(p, (n,)).copy()


class RefPipeline:
    """The reference CPU path, one batch per step()."""

    def __init__(self, query: str, data: str, update: str, batch_size_ints: int, threads: int = 1):
        os.environ["CGB_REF_THREADS"] = str(threads)  # read once, when the pool is first used
        L = ctypes.CDLL(REF_LIB)
        L.cgbref_open.restype = _vp
        L.cgbref_open.argtypes = [ctypes.c_char_p] * 3 + [_u32, ctypes.c_int]
        for n in ["num_batches", "num_updates", "dv_count", "num_dir", "qv", "qe"]:
            getattr(L, "cgbref_" + n).restype = _u32
            getattr(L, "cgbref_" + n).argtypes = [_vp]
        L.cgbref_step.argtypes = [_vp]
        L.cgbref_close.argtypes = [_vp]
        L.cgbref_set_count.argtypes = [_vp, ctypes.c_int]
        L.cgbref_set_parallel_dfs.argtypes = [_vp, ctypes.c_int]
        for n in ["last_count", "last_seed_rows", "total_count"]:
            getattr(L, "cgbref_" + n).restype = _u64
            getattr(L, "cgbref_" + n).argtypes = [_vp]
        L.cgbref_last_matched.argtypes = [_vp]
        L.cgbref_last_keys.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(_u64p)]
        L.cgbref_last_keys.restype = _u64
        L.cgbref_init_keys.argtypes = [_vp, ctypes.POINTER(_u64p)]
        L.cgbref_init_keys.restype = _u64
        L.cgbref_last_edge_ok.argtypes = [_vp]
        L.cgbref_last_edge_ok.restype = _u8p
        L.cgbref_global_order.argtypes = [_vp, _vp]
        L.cgbref_cardinalities.argtypes = [_vp]
        L.cgbref_cardinalities.restype = ctypes.POINTER(_u32)
        L.cgbref_avg_degrees.argtypes = [_vp]
        L.cgbref_avg_degrees.restype = ctypes.POINTER(ctypes.c_float)
        L.cgbref_indexing_order.argtypes = [_vp, _u32, _vp, _vp, _vp]
        L.cgbref_indexing_order.restype = _u32
        L.cgbref_rebuild_vertices.argtypes = [_vp, _u32]
        L.cgbref_rebuild_vertices.restype = _u32
        L.cgbref_new2old.argtypes = [_vp]
        L.cgbref_new2old.restype = ctypes.POINTER(_u32)
        L.cgbref_dump_main.argtypes = [_vp, _vp, _u64]
        L.cgbref_dump_main.restype = _u64
        L.cgbref_last_times.argtypes = [_vp, _vp]
        L.cgbref_li.argtypes = [_vp, _vp, _u64]
        L.cgbref_li.restype = _u64
        L.cgbref_set_sample_budget.argtypes = [_vp, ctypes.c_double]
        L.cgbref_set_progress.argtypes = [_vp, _vp]
        L.cgbref_last_sample.argtypes = [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                                         ctypes.POINTER(ctypes.c_double)]
        self.L = L
        self.h = L.cgbref_open(query.encode(), data.encode(), update.encode(), batch_size_ints, 1)

    def close(self):
        if self.h:
            self.L.cgbref_close(self.h)
            self.h = None

    @property
    def num_batches(self) -> int:
        return self.L.cgbref_num_batches(self.h)

    @property
    def dv_count(self) -> int:
        return self.L.cgbref_dv_count(self.h)

    @property
    def qe(self) -> int:
        return self.L.cgbref_qe(self.h)

    @property
    def qv(self) -> int:
        return self.L.cgbref_qv(self.h)

    @property
    def num_dir(self) -> int:
        return self.L.cgbref_num_dir(self.h)

    def set_count(self, on: bool) -> None:
        self.L.cgbref_set_count(self.h, 1 if on else 0)

    def set_parallel_dfs(self, on: bool) -> None:
        self.L.cgbref_set_parallel_dfs(self.h, 1 if on else 0)

    def set_sample_budget(self, ms: float) -> None:
        self.L.cgbref_set_sample_budget(self.h, float(ms))

    def last_sample(self) -> tuple[int, int, float]:
        d, t, ms = _u64(0), _u64(0), ctypes.c_double(0)
        self.L.cgbref_last_sample(self.h, ctypes.byref(d), ctypes.byref(t), ctypes.byref(ms))
        return d.value, t.value, ms.value

    def init_keys(self) -> np.ndarray:
        p = _u64p()
        n = self.L.cgbref_init_keys(self.h, ctypes.byref(p))
        return _as_np(p, n)

    def global_order(self) -> np.ndarray:
        o = (ctypes.c_uint8 * 12)()
        self.L.cgbref_global_order(self.h, o)
        return np.array(list(o)[: self.qv], dtype=np.uint8)

    def cardinalities(self) -> np.ndarray:
        p = self.L.cgbref_cardinalities(self.h)
        return np.array([p[i] for i in range(self.num_dir)], dtype=np.uint32)

    def avg_degrees(self) -> np.ndarray:
        p = self.L.cgbref_avg_degrees(self.h)
        return np.array([p[i] for i in range(self.num_dir)], dtype=np.float32)

    def indexing_order(self, ei: int):
        vs = np.zeros(12, np.uint8)
        offs = np.zeros(13, np.uint8)
        bni = np.zeros(160, np.uint8)
        n = self.L.cgbref_indexing_order(self.h, ei, vs.ctypes.data, offs.ctypes.data, bni.ctypes.data)
        return vs[: self.qv].copy(), offs[: self.qv + 1].copy(), bni[:n].copy()

    def rebuild_vertices(self, ei: int) -> int:
        return int(self.L.cgbref_rebuild_vertices(self.h, ei))

    def new2old(self) -> np.ndarray:
        n = self.dv_count
        p = self.L.cgbref_new2old(self.h)
        return np.ctypeslib.as_array(p, (n,)).copy() if n else np.zeros(0, np.uint32)

    def step(self) -> int:
        return self.L.cgbref_step(self.h)

    def last(self) -> dict:
        p = _u64p()
        keys = []
        for w in range(3):
            n = self.L.cgbref_last_keys(self.h, w, ctypes.byref(p))
            keys.append(_as_np(p, n))
        okp = self.L.cgbref_last_edge_ok(self.h)
        qe = self.qe
        t = (ctypes.c_double * 4)()
        self.L.cgbref_last_times(self.h, t)
        return {
            "ins": keys[0], "del": keys[1], "delta": keys[2],
            "edge_ok": np.array([okp[i] for i in range(qe)], dtype=np.uint8) if okp else np.zeros(qe, np.uint8),
            "dv": self.dv_count, "count": self.L.cgbref_last_count(self.h),
            "matched": bool(self.L.cgbref_last_matched(self.h)),
            "times_ms": {"s1": t[0], "staging": t[1], "mirror": t[2], "match": t[3]},
        }

    def dump_main_original_ids(self) -> np.ndarray:
        n = self.L.cgbref_dump_main(self.h, None, 0)
        out = np.zeros(max(n, 1), dtype=np.uint64)
        self.L.cgbref_dump_main(self.h, out.ctypes.data, n)
        return out[:n]

    def li(self) -> np.ndarray:
        n = self.L.cgbref_li(self.h, None, 0)
        out = np.zeros(max(n, 1), dtype=np.uint32)
        self.L.cgbref_li(self.h, out.ctypes.data, n)
        return out[:n]


class Oracle:
    """Plain-C restatement of the per-batch path (oracle/oracle.c)."""

    def __init__(self, qv: int, edges):
        L = ctypes.CDLL(ORACLE_LIB)
        L.orc_create.restype = _vp
        L.orc_create.argtypes = [_u32, _u32, _vp]
        L.orc_destroy.argtypes = [_vp]
        L.orc_build.argtypes = [_vp, _vp, _u64, _u32]
        L.orc_build.restype = ctypes.c_int
        L.orc_batch.restype = _u64
        L.orc_batch.argtypes = [_vp, _u32, _vp, _u64, _vp, _u64, _vp, _u64, _vp, ctypes.c_int, _vp]
        L.orc_dump.restype = _u64
        L.orc_dump.argtypes = [_vp, _vp, _u64]
        L.orc_asymmetry.restype = _u64
        L.orc_asymmetry.argtypes = [_vp]
        L.orc_edge_counts.argtypes = [_vp, _vp]
        L.orc_num_edges.argtypes = [_vp]
        L.orc_num_edges.restype = _u32
        L.orc_dir.argtypes = [_vp, _u32, _u32]
        L.orc_dir.restype = _u32
        L.orc_starting_edge.argtypes = [_vp, _vp, _vp, _vp]
        L.orc_set_valid_bits.argtypes = [_vp, ctypes.c_int, _u32, _u32]
        L.orc_valid_bits.argtypes = [_vp, _vp, _u64]
        L.orc_valid_bits.restype = _u64
        L.orc_indexing_order.argtypes = [_vp, _u32, _u32, _u32, _vp, _vp, _vp, _vp]
        L.orc_indexing_order.restype = _u32
        L.orc_set_shard.argtypes = [_vp, _u32, _u32, _vp]
        L.orc_bruteforce.restype = _u64
        L.orc_bruteforce.argtypes = [_u32, _vp, _vp, _vp, _u32, _vp, _u32, _vp]
        self.L = L
        e = np.asarray(edges, dtype=np.uint32).reshape(-1)
        self.h = L.orc_create(qv, len(e) // 2, e.ctypes.data)
        if not self.h:
            raise ValueError("bad query")
        self.qe = L.orc_num_edges(self.h)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build(self, keys: np.ndarray, dv: int) -> None:
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        if self.L.orc_build(self.h, keys.ctypes.data if len(keys) else None, len(keys), dv) != 0:
            raise ValueError("bad initial keys")

    def batch(self, dv: int, ins, dele, delta, edge_ok: Optional[np.ndarray] = None, mode: int = PER_EDGE,
              global_order: Optional[np.ndarray] = None) -> int:
        arrs = [np.ascontiguousarray(a, dtype=np.uint64) for a in (ins, dele, delta)]
        ok = None if edge_ok is None else np.ascontiguousarray(edge_ok, dtype=np.uint8)
        go = None if global_order is None else np.ascontiguousarray(global_order, dtype=np.uint8)
        r = self.L.orc_batch(self.h, dv, *[x for a in arrs for x in (a.ctypes.data if len(a) else None, len(a))],
                             ok.ctypes.data if ok is not None else None, mode,
                             go.ctypes.data if go is not None else None)
        if r == 2**64 - 1:
            raise ValueError("bad batch keys")
        return int(r)

    def edge_counts(self) -> np.ndarray:
        out = np.zeros(16, dtype=np.uint64)
        self.L.orc_edge_counts(self.h, out.ctypes.data)
        return out[: self.qe]

    def dump(self) -> np.ndarray:
        n = self.L.orc_dump(self.h, None, 0)
        out = np.zeros(max(n, 1), dtype=np.uint64)
        self.L.orc_dump(self.h, out.ctypes.data, n)
        return out[:n]

    def starting_edge(self, card: np.ndarray, avg: np.ndarray) -> tuple[int, int]:
        c = np.ascontiguousarray(card, dtype=np.uint32)
        a = np.ascontiguousarray(avg, dtype=np.float32)
        out = np.zeros(2, np.uint32)
        self.L.orc_starting_edge(self.h, c.ctypes.data, a.ctypes.data, out.ctypes.data)
        return int(out[0]), int(out[1])

    def indexing_order(self, ei: int, start: tuple[int, int]):
        """(vs, offsets, bni, rebuild-vertex mask or ~0) of query edge ei."""
        vs = np.zeros(12, np.uint8)
        offs = np.zeros(13, np.uint8)
        bni = np.zeros(160, np.uint8)
        vf = _u32(0)
        n = self.L.orc_indexing_order(self.h, ei, start[0], start[1], vs.ctypes.data, offs.ctypes.data,
                                      bni.ctypes.data, ctypes.byref(vf))
        return vs, offs, bni[:n].copy(), int(vf.value)

    def set_valid_bits(self, mode: int, start: tuple[int, int]) -> None:
        """mode 0 = off, 1 = compute per matched batch, 2 = compute and prune the count."""
        self.L.orc_set_valid_bits(self.h, mode, start[0], start[1])

    def valid_bits(self) -> np.ndarray:
        n = self.L.orc_valid_bits(self.h, None, 0)
        if n == 2**64 - 1:
            raise ValueError("rebuild flags inconsistent (the reference stops here)")
        out = np.zeros(max(n, 1), np.uint32)
        self.L.orc_valid_bits(self.h, out.ctypes.data, n)
        return out[:n]

    def set_shard(self, shard: int, num_shards: int, anchor=None) -> None:
        """Counts only the seeds of one shard: those whose key (query edge ei,
        data vertex at query vertex anchor[ei]; default ei's first endpoint)
        hashes to `shard` like the engine's seed groups."""
        a = None if anchor is None else np.ascontiguousarray(anchor, dtype=np.uint8)
        self.L.orc_set_shard(self.h, shard, num_shards, a.ctypes.data if a is not None else None)

    def asymmetry(self) -> int:
        return int(self.L.orc_asymmetry(self.h))

    def bruteforce(self, n: int, edges: np.ndarray, glabels: np.ndarray, qlabels, qedges) -> int:
        """Label-preserving injective embeddings of the query in the graph (n, undirected edges)."""
        e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
        src = np.concatenate([e[:, 0], e[:, 1]])
        dst = np.concatenate([e[:, 1], e[:, 0]])
        order = np.lexsort((dst, src))
        src, dst = src[order], dst[order]
        off = np.zeros(n + 1, dtype=np.uint64)
        np.add.at(off, src + 1, 1)
        off = np.cumsum(off).astype(np.uint64)
        adj = dst.astype(np.uint32)
        gl = np.ascontiguousarray(glabels, dtype=np.uint32)
        ql = np.ascontiguousarray(qlabels, dtype=np.uint32)
        qe = np.ascontiguousarray(np.asarray(qedges, dtype=np.uint32).reshape(-1))
        return int(self.L.orc_bruteforce(n, off.ctypes.data, adj.ctypes.data if len(adj) else None,
                                         gl.ctypes.data, len(ql), ql.ctypes.data, len(qe) // 2, qe.ctypes.data))


def read_graph(path: str) -> tuple[int, np.ndarray, np.ndarray]:
    """Reads a reference-format data graph: (n, labels[n], edges[m,2])."""
    labels = []
    edges = []
    for line in open(path):
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            labels.append(int(t[2]))
        elif t[0] == "e":
            edges.append((int(t[1]), int(t[2])))
    return len(labels), np.array(labels, dtype=np.uint32), np.array(edges, dtype=np.int64).reshape(-1, 2)


def read_updates(path: str) -> np.ndarray:
    out = []
    for line in open(path):
        t = line.split()
        if len(t) >= 3:
            out.append((int(t[1]), int(t[2])))
    return np.array(out, dtype=np.int64).reshape(-1, 2)


# ---------------------------------------------------------------------------
# Supervised sample of the reference CPU path (bench.py's reference arm and
# cpu_baseline): the reference enumerates every embedding, and one seed row on
# an R-MAT hub can run for hours, so the batch runs in a child process that
# publishes progress in shared memory and is stopped at a deadline.
# ---------------------------------------------------------------------------
def _supervised_child(query, data, update, batch_size_ints, threads, shm_name):
    from multiprocessing import shared_memory

    os.environ["CGB_REF_THREADS"] = str(threads)
    shm = shared_memory.SharedMemory(name=shm_name)
    buf = np.ndarray((8,), dtype=np.uint64, buffer=shm.buf)
    ref = RefPipeline(query, data, update, batch_size_ints, threads=threads)
    ref.L.cgbref_set_progress(ref.h, buf.ctypes.data)
    buf[7] = 1
    ref.step()
    buf[7] = 2
    del buf
    shm.close()


def supervised_reference_batch(query: str, data: str, update: str, batch_size_ints: int, threads: int,
                               count_budget_s: float, open_timeout_s: float = 300.0) -> dict:
    """Runs batch 0 of the reference CPU path with all `threads`; Stage 1,
    staging and the mirror update are timed fully, the count for at most
    count_budget_s.  Returns the stage times (ms), rows counted / total and
    the count time spent."""
    import multiprocessing as mp
    import time
    from multiprocessing import shared_memory

    shm = shared_memory.SharedMemory(create=True, size=64)
    buf = np.ndarray((8,), dtype=np.uint64, buffer=shm.buf)
    buf[:] = 0
    ctx = mp.get_context("spawn")
    p = ctx.Process(target=_supervised_child, args=(query, data, update, batch_size_ints, threads, shm.name))
    t0 = time.time()
    p.start()
    try:
        while buf[6] < 2 and p.is_alive() and time.time() - t0 < open_timeout_s:
            time.sleep(0.05)
        t_count = time.time()
        while buf[6] < 3 and p.is_alive() and time.time() - t_count < count_budget_s:
            time.sleep(0.05)
        if buf[6] < 2:
            raise RuntimeError(f"reference child stopped before counting (exit code {p.exitcode})")
        out = {"s1_ms": buf[2] / 1e3, "staging_ms": buf[3] / 1e3, "mirror_ms": buf[4] / 1e3,
               "rows_done": int(buf[0]), "rows_total": int(buf[1]),
               "count_ms": (time.time() - t_count) * 1e3 if buf[6] < 3 else buf[5] / 1e3,
               "finished": bool(buf[6] >= 3), "reached_count": bool(buf[6] >= 2),
               "wall_s": time.time() - t0}
    finally:
        if p.is_alive():
            p.terminate()
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
            p.join(timeout=30)
        del buf
        shm.close()
        shm.unlink()
    return out
