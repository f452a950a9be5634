"""Multi-query engine (cgb_mq_*, through the C ABI) against the reference and
the single-query pipeline.

The engine keeps one data-graph index keyed by target-vertex label and
matches every registered query per batch in one launch.  Its per-batch count
for a query must equal, bit for bit:
  * the reference's own CPU path (oracle/_ref: CaLiG + cpu_dfs) on the same
    seeded stream,
  * the single-query engine fed by the CaLiG producer (the plain pipeline,
    one query per launch), for every query of a mixed set,
  * the same query registered alone (alone vs in the mix),
  * brute-force embedding differences for deletion batches and for dense
    patterns with more than 16 edges (beyond the reference's key encoding).
"""
import os

import numpy as np
import pytest

from cgbdsm_b200 import Engine, MultiQuery, Producer
from cgbdsm_b200.engine import MQ_FLAG_NO_AUTOTUNE, MQ_FLAG_NO_GRAPH
from cgbdsm_b200.workloads import SPECS, GraphData, materialize, read_query
from oracle import bind

pytestmark = pytest.mark.gpu


def write_query(path, labels, edges):
    with open(path, "w") as f:
        for i, lb in enumerate(labels):
            f.write(f"v {i} {lb}\n")
        for a, b in edges:
            f.write(f"e {a} {b} 0\n")


def plain_pipeline_counts(spec, paths, qpath):
    """Per-batch counts of the plain pipeline (CaLiG producer + single-query engine)."""
    ql, qe = read_query(qpath)
    prod = Producer(qpath, paths["data"], paths["update"], spec.cli_batch_size)
    init, dv = prod.initial()
    eng = Engine(dfs_budget_ms=120000)
    eng.load_query(len(ql), qe, ql)
    eng.build_index(init, dv)
    out = []
    for _ in range(prod.num_batches):
        r = prod.next()
        out.append(eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"]))
    eng.close()
    prod.close()
    return out


def mq_counts(g, queries, flags=0):
    m = MultiQuery(flags=flags, dfs_budget_ms=120000)
    m.load_graph(g.labels, g.initial)
    ids = [m.register(len(ql), qe, ql) for ql, qe in queries]
    out = []
    for b in g.batches():
        pos, neg = m.apply_batch(ins=b)
        assert not neg.any()
        out.append([int(pos[i]) for i in ids])
    m.close()
    return out


@pytest.mark.parametrize("name", ["t_tiny", "t_er5", "t_er_sparse", "t_er_tree", "t_rmat", "c1_q25", "t_er_tree_s",
                                  "t_rmat_tree"])
def test_mq_matches_reference_cpu_path(name, workdir):
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ql, qe = read_query(p["query"])
    g = GraphData(spec)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    want = []
    while ref.step() >= 0:
        want.append(ref.last()["count"])
    ref.close()
    got = [c[0] for c in mq_counts(g, [(ql, qe)])]
    assert got == want


def _mixed_queries(g, sizes, shapes, seeds, max_qedges=16):
    out = []
    for size, shape, seed in zip(sizes, shapes, seeds):
        q = g.query(shape, size, seed, max_qedges)
        if q is not None:
            out.append(q)
    return out


@pytest.mark.parametrize("name", ["t_rmat", "t_er6"])
def test_mq_mixed_set_equals_each_query_alone(name, workdir, tmp_path):
    """A mixed set of tree / sparse / dense patterns of 4-8 vertices, matched
    together in one launch, gives every query the counts it gets alone in
    the multi-query engine and alone in the plain pipeline (CaLiG producer +
    single-query engine), batch by batch."""
    spec = SPECS[name]
    p = materialize(spec, workdir)
    g = GraphData(spec)
    rng = np.random.default_rng(5)
    sizes = [int(x) for x in rng.integers(4, 9, 12)]
    shapes = [i % 3 for i in range(12)]
    queries = _mixed_queries(g, sizes, shapes, range(500, 512))
    assert len(queries) >= 8
    mixed = mq_counts(g, queries)
    for i, (ql, qe) in enumerate(queries):
        alone = [c[0] for c in mq_counts(g, [(ql, qe)], flags=MQ_FLAG_NO_AUTOTUNE | MQ_FLAG_NO_GRAPH)]
        assert [c[i] for c in mixed] == alone, f"query {i}: mixed != alone"
        qpath = str(tmp_path / f"q{i}.graph")
        write_query(qpath, ql, qe)
        assert alone == plain_pipeline_counts(spec, p, qpath), f"query {i}: multi-query != plain pipeline"
    assert any(sum(c) for c in mixed)


def test_mq_register_and_unregister_between_batches():
    """Queries join and leave between batches; a query's counts from the batch
    it joined on equal its counts when registered from the start."""
    spec = SPECS["t_rmat"]
    g = GraphData(spec)
    qs = _mixed_queries(g, [5, 6, 5], [0, 1, 2], [900, 901, 902])
    full = mq_counts(g, qs, flags=MQ_FLAG_NO_AUTOTUNE)
    m = MultiQuery(dfs_budget_ms=120000)
    m.load_graph(g.labels, g.initial)
    ids = {0: m.register(len(qs[0][0]), qs[0][1], qs[0][0])}
    for b, batch in enumerate(g.batches()):
        if b == 2:
            ids[1] = m.register(len(qs[1][0]), qs[1][1], qs[1][0])
        if b == 3:
            m.unregister(ids.pop(0))
            ids[2] = m.register(len(qs[2][0]), qs[2][1], qs[2][0])
        pos, _ = m.apply_batch(ins=batch)
        for k, qid in ids.items():
            assert int(pos[qid]) == full[b][k], f"batch {b} query {k}"
    m.close()


def _bruteforce(o, n, edges, labels, ql, qe):
    return o.bruteforce(n, np.asarray(edges, dtype=np.int64).reshape(-1, 2), labels, ql, qe)


def test_mq_deletions_count_destroyed_embeddings():
    """Batches that delete and insert: negative matches = embeddings the
    deletions destroy, |Emb(G)| - |Emb(G - del)|; positive = |Emb(G - del +
    ins)| - |Emb(G - del)|; absent deletions, repeated and already present
    insertions change nothing.  Brute force on a small graph."""
    rng = np.random.default_rng(3)
    n = 120
    labels = rng.integers(0, 3, n).astype(np.uint32)
    pairs = set()
    while len(pairs) < 700:
        a, b = (int(x) for x in rng.integers(0, n, 2))
        if a != b:
            pairs.add((min(a, b), max(a, b)))
    edges = sorted(pairs)
    cur = set(edges[:600])
    pool = edges[600:]
    queries = [([0, 1, 2], [(0, 1), (1, 2), (0, 2)]), ([0, 1, 1, 2], [(0, 1), (0, 2), (1, 3), (2, 3)]),
               ([1, 0, 2, 0, 1], [(0, 1), (1, 2), (2, 3), (3, 4)])]
    m = MultiQuery(dfs_budget_ms=60000)
    m.load_graph(labels, sorted(cur))
    ids = [m.register(len(ql), qe, ql) for ql, qe in queries]
    o = bind.Oracle(3, [(0, 1), (1, 2)])
    for b in range(6):
        dels = [e for e in sorted(cur) if rng.random() < 0.05]
        dels += [(0, 1), (2, 3)] if (0, 1) not in cur else []  # possibly absent deletions
        ins = [pool.pop() for _ in range(min(len(pool), 12))]
        ins += ins[:2] + [next(iter(cur))]  # repeats and an edge already present
        before = [_bruteforce(o, n, sorted(cur), labels, ql, qe) for ql, qe in queries]
        mid_set = cur - set(dels)
        mid = [_bruteforce(o, n, sorted(mid_set), labels, ql, qe) for ql, qe in queries]
        after_set = mid_set | set((min(a, b), max(a, b)) for a, b in ins)
        after = [_bruteforce(o, n, sorted(after_set), labels, ql, qe) for ql, qe in queries]
        pos, neg = m.apply_batch(ins=ins, dele=dels)
        for k, qid in enumerate(ids):
            assert int(neg[qid]) == before[k] - mid[k], f"batch {b} query {k}: negative"
            assert int(pos[qid]) == after[k] - mid[k], f"batch {b} query {k}: positive"
        cur = after_set
    m.close()


def test_mq_dense_patterns_beyond_sixteen_edges():
    """Dense 11- and 12-vertex patterns (17+ edges, beyond the reference's
    5-bit directed query-edge encoding) on a dense small graph, against brute
    force: the sum of batch counts equals |Emb(G_final)| - |Emb(G_initial)|
    and every batch's count equals its own difference."""
    rng = np.random.default_rng(17)
    n = 30
    labels = rng.integers(0, 2, n).astype(np.uint32)
    allp = [(a, b) for a in range(n) for b in range(a + 1, n) if rng.random() < 0.4]
    order = rng.permutation(len(allp))
    allp = [allp[i] for i in order]
    init, stream = allp[: len(allp) - 60], allp[len(allp) - 60:]
    adj = {v: set() for v in range(n)}
    for a, b in allp:
        adj[a].add(b)
        adj[b].add(a)
    queries = []
    for size in (11, 12):
        vs, tree = [0], []
        while len(vs) < size:  # BFS sample: tree edges first, then induced edges up to the target count
            for v in list(vs):
                for w in sorted(adj[v]):
                    if w not in vs and len(vs) < size:
                        vs.append(w)
                        tree.append((vs.index(v), len(vs) - 1))
        extra = [(i, j) for i in range(size) for j in range(i + 1, size)
                 if vs[j] in adj[vs[i]] and (i, j) not in tree]
        qe = sorted(tree + extra[: 17 + size - 11 - len(tree)])
        queries.append(([int(labels[v]) for v in vs], qe))
    for ql, qe in queries:
        assert len(qe) > 16
    m = MultiQuery(dfs_budget_ms=120000)
    m.load_graph(labels, init)
    ids = [m.register(len(ql), qe, ql) for ql, qe in queries]
    o = bind.Oracle(3, [(0, 1), (1, 2)])
    cur = list(init)
    for b in range(0, 60, 20):
        batch = stream[b:b + 20]
        before = [_bruteforce(o, n, cur, labels, ql, qe) for ql, qe in queries]
        cur = cur + batch
        after = [_bruteforce(o, n, cur, labels, ql, qe) for ql, qe in queries]
        pos, _ = m.apply_batch(ins=batch)
        for k, qid in enumerate(ids):
            assert int(pos[qid]) == (after[k] - before[k]) % 2**64, f"batch {b} query {k}"
    m.close()


def test_mq_graph_replay_and_autotune_keep_counts():
    """The matching step replayed as a CUDA graph, the autotuned schedule and
    the plain launches all give the same counts."""
    spec = SPECS["t_rmat"]
    g = GraphData(spec)
    qs = _mixed_queries(g, [5, 6, 7, 5, 6], [0, 1, 2, 2, 0], range(700, 705))
    a = mq_counts(g, qs)
    b = mq_counts(g, qs, flags=MQ_FLAG_NO_AUTOTUNE | MQ_FLAG_NO_GRAPH)
    c = mq_counts(g, qs, flags=MQ_FLAG_NO_AUTOTUNE)
    assert a == b == c
