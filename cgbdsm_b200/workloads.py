"""Seeded synthetic workloads in the reference's text formats.

The reference measures on public graphs that are not available here; these
configurations stand in for them with the shapes, sizes and distributions
the engine is measured on (seeds fixed so every run sees the same input):

  c1  Erdos-Renyi 10,000 vertices / 50,000 edges, 8 uniform labels,
      10% (5,000 edges) held out and re-inserted in batches of 1,000,
      5-vertex dense pattern (densest induced BFS sample, see gen.cpp).
      With query seed 11 no batch has a positive match (the sampled
      occurrence uses no held-out edge, and the pattern is rare at this
      density); c1_q25 is the same graph and stream with query seed 25, the
      first seed whose first two batches have positive matches (4 and 6).
  c2  R-MAT(0.57,0.19,0.19,0.05) 1,000,000 vertices / 10,000,000 edges,
      16 labels Zipf(1.2), 1,000,000 held out, batches of 100,000,
      9-vertex dense pattern with <= 16 edges.  Every sampled pattern is
      centred on an R-MAT hub; query seeds 24-32, 34-39, 42, 43 need more
      than 3 s of matching for the first batch on a B200, seeds 33 and 40
      reach ~2^63 matches per batch (the stream total would wrap the u64
      counter), so seed 41 is used (~1.9e16 matches per batch).
  c3  R-MAT 4,000,000 / 34,000,000, 32 labels Zipf(1.0), 3,400,000 held
      out, batches of 1,000,000, 7-vertex tree and sparse patterns.
Small seeded variants ("t*") are used by the parity tests.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

_HERE = os.path.dirname(os.path.abspath(__file__))
GEN_LIB = os.path.join(_HERE, "libcgbgen.so")


@dataclass(frozen=True)
class WorkloadSpec:
    name: str
    kind: int            # 0 = Erdos-Renyi, 1 = R-MAT
    n: int
    m: int
    labels: int
    zipf: float          # <= 0: uniform labels
    holdout: int
    batch_edges: int     # insertions per batch (reference CLI batch_size = 2x, F2)
    qshape: int          # 0 dense, 1 sparse, 2 tree
    qsize: int
    seed_graph: int
    seed_labels: int
    seed_holdout: int
    seed_query: int
    max_qedges: int = 16

    @property
    def num_batches(self) -> int:
        return (self.holdout + self.batch_edges - 1) // self.batch_edges

    @property
    def cli_batch_size(self) -> int:
        """The reference CLI's [batch_size] counts ints, two per edge (main_calig.cpp:104, F2)."""
        return 2 * self.batch_edges


SPECS = {
    "c1": WorkloadSpec("c1", 0, 10_000, 50_000, 8, 0.0, 5_000, 1_000, 0, 5, 1, 2, 3, 11),
    "c1_q25": WorkloadSpec("c1_q25", 0, 10_000, 50_000, 8, 0.0, 5_000, 1_000, 0, 5, 1, 2, 3, 25),
    "c2": WorkloadSpec("c2", 1, 1_000_000, 10_000_000, 16, 1.2, 1_000_000, 100_000, 0, 9, 21, 22, 23, 41),
    "c3_tree": WorkloadSpec("c3_tree", 1, 4_000_000, 34_000_000, 32, 1.0, 3_400_000, 1_000_000, 2, 7,
                            31, 32, 33, 34),
    "c3_sparse": WorkloadSpec("c3_sparse", 1, 4_000_000, 34_000_000, 32, 1.0, 3_400_000, 1_000_000, 1, 7,
                              31, 32, 33, 35),
    # small parity workloads (CPU oracle finishes in seconds)
    "t_er5": WorkloadSpec("t_er5", 0, 2_000, 40_000, 4, 0.0, 4_000, 500, 0, 5, 101, 102, 103, 7),
    "t_er6": WorkloadSpec("t_er6", 0, 3_000, 60_000, 3, 0.0, 6_000, 1_000, 0, 6, 111, 112, 113, 5),
    "t_er_sparse": WorkloadSpec("t_er_sparse", 0, 3_000, 45_000, 3, 0.0, 4_500, 750, 1, 6, 121, 122, 123, 9),
    "t_er_tree": WorkloadSpec("t_er_tree", 0, 3_000, 30_000, 3, 0.0, 3_000, 600, 2, 5, 131, 132, 133, 13),
    "t_rmat": WorkloadSpec("t_rmat", 1, 8_192, 60_000, 8, 1.0, 6_000, 1_000, 0, 5, 141, 142, 143, 17),
    "t_tiny": WorkloadSpec("t_tiny", 0, 300, 2_400, 2, 0.0, 400, 50, 0, 4, 151, 152, 153, 3),
    # trees whose labels reach the level sums: every query label distinct
    # (dense sums over several positions), or shared with prefix positions
    # (one position, prefix vertices subtracted); R-MAT tree of C3's shape
    "t_er_tree_u": WorkloadSpec("t_er_tree_u", 0, 3_000, 30_000, 12, 0.0, 3_000, 600, 2, 6, 161, 162, 163, 161),
    "t_er_tree_s": WorkloadSpec("t_er_tree_s", 0, 3_000, 30_000, 12, 0.0, 3_000, 600, 2, 6, 161, 162, 163, 160),
    "t_rmat_tree": WorkloadSpec("t_rmat_tree", 1, 8_192, 60_000, 16, 1.0, 6_000, 1_200, 2, 7, 171, 172, 173, 174),
    # the R-MAT 4M/34M stream's label distribution on a small graph (tests
    # run the headline's patterns on it)
    "t_rmat32": WorkloadSpec("t_rmat32", 1, 8_192, 60_000, 32, 1.0, 6_000, 1_200, 1, 7, 181, 182, 183, 184),
}


def _gen():
    if not os.path.exists(GEN_LIB):
        raise FileNotFoundError(f"{GEN_LIB} not built; run `python -m cgbdsm_b200.build`")
    lib = ctypes.CDLL(GEN_LIB)
    f = lib.cgbgen_workload
    f.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_uint32, ctypes.c_double,
                                          ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                          ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_uint32)]
    return f


def materialize(spec: WorkloadSpec, directory: str) -> dict[str, str]:
    """Writes data.graph, update.graph and query.graph for spec (cached by name)."""
    d = os.path.join(directory, spec.name)
    paths = {k: os.path.join(d, f"{k}.graph") for k in ("data", "update", "query")}
    stamp = os.path.join(d, "spec.txt")
    if all(os.path.exists(p) for p in paths.values()) and os.path.exists(stamp):
        if open(stamp).read() == repr(spec):
            return paths
    os.makedirs(d, exist_ok=True)
    qe = ctypes.c_uint32(0)
    rc = _gen()(paths["data"].encode(), paths["update"].encode(), paths["query"].encode(), spec.kind, spec.n,
                spec.m, 0.57, 0.19, 0.19, spec.labels, spec.zipf, spec.holdout, spec.seed_graph,
                spec.seed_labels, spec.seed_holdout, spec.qshape, spec.qsize, spec.max_qedges, spec.seed_query,
                ctypes.byref(qe))
    if rc != 0:
        raise RuntimeError(f"workload generation failed for {spec.name}: rc={rc}")
    with open(stamp, "w") as f:
        f.write(repr(spec))
    return paths


def materialize_query(spec: WorkloadSpec, path: str, seed_query: int) -> int:
    """Writes only the query pattern of spec with another query seed (graph
    and stream are regenerated in memory, not written).  Returns its edge count."""
    qe = ctypes.c_uint32(0)
    rc = _gen()(None, None, path.encode(), spec.kind, spec.n, spec.m, 0.57, 0.19, 0.19, spec.labels, spec.zipf,
                spec.holdout, spec.seed_graph, spec.seed_labels, spec.seed_holdout, spec.qshape, spec.qsize,
                spec.max_qedges, seed_query, ctypes.byref(qe))
    if rc != 0:
        raise RuntimeError(f"query generation failed: rc={rc}")
    return qe.value


class GraphData:
    """A workload's graph in memory (cgbgen_open): labels, initial edges and
    the held-out stream as (x, y) pairs, identical to what materialize()
    writes, plus query patterns sampled from the final graph (query seed s
    gives the pattern materialize() writes with seed_query s)."""

    def __init__(self, spec: WorkloadSpec):
        import numpy as np

        lib = ctypes.CDLL(GEN_LIB)
        lib.cgbgen_open.restype = ctypes.c_void_p
        lib.cgbgen_open.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64,
                                    ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
        lib.cgbgen_close.argtypes = [ctypes.c_void_p]
        lib.cgbgen_sizes.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.cgbgen_copy.argtypes = [ctypes.c_void_p] * 4
        lib.cgbgen_query.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]
        self.lib = lib
        self.spec = spec
        self.h = lib.cgbgen_open(spec.kind, spec.n, spec.m, 0.57, 0.19, 0.19, spec.labels, spec.zipf, spec.holdout,
                                 spec.seed_graph, spec.seed_labels, spec.seed_holdout)
        sz = np.zeros(3, dtype=np.uint64)
        lib.cgbgen_sizes(self.h, sz.ctypes.data)
        self.n = int(sz[0])
        self.labels = np.zeros(self.n, dtype=np.uint32)
        self.initial = np.zeros((int(sz[1]), 2), dtype=np.uint32)
        self.stream = np.zeros((int(sz[2]), 2), dtype=np.uint32)
        lib.cgbgen_copy(self.h, self.labels.ctypes.data, self.initial.ctypes.data, self.stream.ctypes.data)

    def query(self, shape: int, size: int, seed: int, max_qedges: int = 32):
        """(labels, edges) of a pattern: shape 0 dense, 1 sparse, 2 tree; None if none was found."""
        import numpy as np

        lab = np.zeros(12, dtype=np.uint32)
        edges = np.zeros(2 * 66, dtype=np.uint32)
        qv, qe = ctypes.c_uint32(0), ctypes.c_uint32(0)
        rc = self.lib.cgbgen_query(self.h, shape, size, max_qedges, seed, lab.ctypes.data, edges.ctypes.data,
                                   ctypes.byref(qv), ctypes.byref(qe))
        if rc != 0:
            return None
        return [int(x) for x in lab[: qv.value]], [(int(edges[2 * i]), int(edges[2 * i + 1])) for i in range(qe.value)]

    def batches(self):
        """The stream cut into the spec's batches."""
        b = self.spec.batch_edges
        return [self.stream[i:i + b] for i in range(0, len(self.stream), b)]

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cgbgen_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_query(path: str) -> tuple[list[int], list[tuple[int, int]]]:
    labels: dict[int, int] = {}
    edges: list[tuple[int, int]] = []
    for line in open(path):
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            labels[int(t[1])] = int(t[2])
        elif t[0] == "e":
            edges.append((int(t[1]), int(t[2])))
    return [labels[i] for i in range(len(labels))], edges


def write_binary_csr(spec: WorkloadSpec, directory: str, nvcls: int) -> dict[str, str]:
    """Writes the full graph of spec (initial edges plus the held-out stream)
    as the reference's binary CSR prefix (calig.cpp:218-323): <prefix>.meta.txt
    ("n m 4 8 0 0 maxdeg 0 nvcls 0"), <prefix>.vertex.bin (u64 row pointers),
    <prefix>.edge.bin (u32 neighbours, both directions, rows sorted).  Labels
    and the update stream are not stored: the reader draws them.  Returns
    {"data": prefix, "query": path of spec's query}."""
    import numpy as np

    p = materialize(spec, directory)
    n = 0
    edges = []
    for path in (p["data"], p["update"]):
        for line in open(path):
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                n = max(n, int(t[1]) + 1)
            elif len(t) >= 3:
                edges.append((int(t[1]), int(t[2])))
    e = np.array(edges, dtype=np.int64).reshape(-1, 2)
    both = np.concatenate([e, e[:, ::-1]])
    both = np.unique(both, axis=0)  # sorted by (row, neighbour), duplicates dropped
    deg = np.bincount(both[:, 0], minlength=n)
    row = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(deg, out=row[1:])
    prefix = os.path.join(directory, spec.name, f"{spec.name}_csr")
    with open(prefix + ".meta.txt", "w") as f:
        f.write(f"{n} {len(both)} 4 8 0 0 {int(deg.max()) if n else 0} 0 {nvcls} 0\n")
    row.tofile(prefix + ".vertex.bin")
    both[:, 1].astype(np.uint32).tofile(prefix + ".edge.bin")
    return {"data": prefix, "query": p["query"]}
