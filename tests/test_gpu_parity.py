"""GPU parity: the engine (through the C ABI) against the oracle.

Counts and index contents must be bit-exact:
  * against the reference's own CPU path (oracle/_ref) on seeded workloads,
  * against the C restatement (oracle/oracle.c) on random key streams and on
    the edge cases the reference's pipeline has (empty delta, vertex-id growth,
    duplicate inserts, removal of absent keys, invalid keys).
"""
import numpy as np
import pytest

from cgbdsm_b200 import CgbError, Engine
from cgbdsm_b200.engine import (FLAG_ENUMERATE_TAIL, FLAG_FORCE_SPLIT, FLAG_MASK_PRUNE, FLAG_NO_RUN_BITS,
                                FLAG_NO_SEED_GROUPS, FLAG_NO_TAIL_CACHE, FLAG_PLAIN_CORE_ORDER, FLAG_VALID_BITS,
                                FLAG_NO_LEVEL_SUM, FLAG_WARP_TAIL)
from cgbdsm_b200.workloads import SPECS, materialize, read_query
from oracle import bind

pytestmark = pytest.mark.gpu

PIPELINE_CASES = ["t_tiny", "t_er5", "t_er6", "t_er_sparse", "t_er_tree", "t_rmat", "c1", "c1_q25", "t_er_tree_u",
                  "t_er_tree_s", "t_rmat_tree"]


def _key(d, u, v):
    return (np.uint64(d) << np.uint64(59)) | (np.uint64(u) << np.uint64(32)) | np.uint64(v)


@pytest.mark.parametrize("flags", [0, FLAG_ENUMERATE_TAIL, FLAG_FORCE_SPLIT | FLAG_ENUMERATE_TAIL, FLAG_FORCE_SPLIT,
                                   FLAG_NO_TAIL_CACHE, FLAG_NO_SEED_GROUPS, FLAG_NO_RUN_BITS, FLAG_PLAIN_CORE_ORDER,
                                   FLAG_WARP_TAIL, FLAG_NO_LEVEL_SUM | FLAG_FORCE_SPLIT],
                         ids=["counted_tail", "enumerated_tail", "stolen_enumerated", "stolen_counted",
                              "counted_no_prefix_cache", "seed_per_dfs", "searched_runs", "greedy_core_order",
                              "warp_tail", "no_level_sum_stolen"])
@pytest.mark.parametrize("name", PIPELINE_CASES)
def test_engine_matches_reference_cpu_path(name, flags, workdir):
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    qlabels, qedges = read_query(p["query"])
    eng = Engine(flags=flags)
    eng.load_query(len(qlabels), qedges, qlabels)
    orc = bind.Oracle(len(qlabels), qedges)
    init = ref.init_keys()
    eng.build_index(init, ref.dv_count)
    orc.build(init, ref.dv_count)
    assert np.array_equal(eng.read_index(), orc.dump())
    nb = 0
    while ref.step() >= 0:
        r = ref.last()
        c = eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
        co = orc.batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"], bind.PER_EDGE)
        assert c == r["count"], f"{name} batch {nb}: engine {c} != reference {r['count']}"
        assert np.array_equal(eng.edge_counts(), orc.edge_counts())
        assert co == c
        nb += 1
    assert np.array_equal(eng.read_index(), orc.dump())
    ref.close()
    eng.close()


def _random_query(rng, qv, extra):
    edges = set()
    for v in range(1, qv):  # spanning tree
        edges.add((int(rng.integers(0, v)), v))
    cand = [(a, b) for a in range(qv) for b in range(a + 1, qv) if (a, b) not in edges]
    rng.shuffle(cand)
    for e in cand[:extra]:
        edges.add(e)
    return sorted(edges)


def _sym_keys(orc, pairs_by_edge):
    """pairs_by_edge: list of (a, b, x, y) = query edge (a,b) realised by data edge (x,y)."""
    ks = []
    for a, b, x, y in pairs_by_edge:
        ks.append(_key(orc.L.orc_dir(orc.h, a, b), x, y))
        ks.append(_key(orc.L.orc_dir(orc.h, b, a), y, x))
    return np.array(ks, dtype=np.uint64) if ks else np.zeros(0, np.uint64)


@pytest.mark.parametrize("seed", range(8))
def test_random_symmetric_streams(seed):
    _random_stream(seed, 0.0)


@pytest.mark.parametrize("seed", range(4))
def test_random_streams_with_self_loops(seed):
    """Self-loop keys (x, x) never complete an embedding (injectivity) but do
    change the counted tails: a matched vertex then lies in its own list and
    must be excluded from it."""
    _random_stream(100 + seed, 0.15)


@pytest.mark.parametrize("name", PIPELINE_CASES)
def test_every_run_bitset_matches_reference(name, workdir, monkeypatch):
    """Long runs are tested through per-batch bit sets (DFS probes and tail
    counts); with the length threshold at 1 every run has one.  Counts and
    index stay the reference's."""
    monkeypatch.setenv("CGB_RUN_BITS_MIN_LEN", "1")
    test_engine_matches_reference_cpu_path(name, FLAG_FORCE_SPLIT if name == "t_rmat" else 0, workdir)


@pytest.mark.parametrize("seed", range(6))
def test_every_run_bitset_random_streams(seed, monkeypatch):
    monkeypatch.setenv("CGB_RUN_BITS_MIN_LEN", "1")
    _random_stream(300 + seed, 0.1 if seed % 2 else 0.0, nlabels=seed % 4)


@pytest.mark.parametrize("seed", range(12))
def test_random_labelled_streams(seed):
    """Labelled queries with pendant vertices: seed edges with a pendant
    endpoint run one DFS per seed group (the other endpoint), each embedding
    weighted by the group's seeds it does not reuse; the keys respect the
    labels (as the producer's candidate lists do), self-loops included.
    Every other seed also runs with one DFS per seed."""
    _random_stream(200 + seed, 0.1 if seed % 3 == 2 else 0.0, nlabels=1 + seed % 3)


@pytest.mark.parametrize("seed", range(6))
def test_pendant_with_same_label_tail(seed):
    """A hub with a pendant and a second degree-1 neighbour of the pendant's
    label: the grouped plan keeps that neighbour as a counted tail and
    subtracts, per embedding, the seeds that are its candidates."""
    query = (5, [(0, 1), (0, 2), (0, 3), (0, 4), (3, 4)], [0, 1, 1, 2, 3])
    _random_stream(400 + seed, 0.1 if seed % 2 else 0.0, nlabels=4, query=query)


def _random_stream(seed, self_loop_rate, nlabels=0, query=None):
    rng = np.random.default_rng(1000 + seed)
    qv = int(rng.integers(3, 7))
    qedges = _random_query(rng, qv, int(rng.integers(0, 4)))
    if query is not None:
        qv, qedges = query[0], query[1]
    dv0 = 60
    flags = FLAG_FORCE_SPLIT if seed % 2 else 0
    if nlabels and seed % 4 >= 2:
        flags |= FLAG_NO_SEED_GROUPS
    eng = Engine(flags=flags)
    orc = bind.Oracle(qv, qedges)
    if nlabels:
        # labels: query vertices and data vertices drawn from nlabels values;
        # a key (a -> b, x, y) only pairs x of a's label with y of b's label
        qlab = [int(x) for x in rng.integers(0, nlabels, qv)]
        if query is not None:
            qlab = list(query[2])
        eng.load_query(qv, qedges, qlab)
        dlab = rng.integers(0, nlabels, 4096)
        dlab[:2 * nlabels] = np.arange(2 * nlabels) % nlabels  # hubs 0 .. 2*nlabels-1 cover every label
    else:
        eng.load_query(qv, qedges)

    def pick(dv, lab, avoid=-1):
        while True:
            x = int(rng.integers(0, dv))
            if x != avoid and (not nlabels or dlab[x] == lab):
                return x

    def rand_pairs(n, dv):
        # a third of the pairs touch a hub (vertex 0 or 1, or per label), so
        # some lists are long enough (> 96) for the DFS to split them through
        # the work queue
        out = []
        for _ in range(n):
            a, b = qedges[int(rng.integers(0, len(qedges)))]
            if nlabels:
                if rng.random() < 0.5:
                    a, b = b, a
                la, lb = qlab[a], qlab[b]
                x = pick(dv, la)
                if rng.random() < 0.33:
                    x = la + nlabels * int(rng.integers(0, 2))
                if rng.random() < self_loop_rate and la == lb:
                    y = x
                else:
                    y = pick(dv, lb, avoid=x)
            else:
                x, y = rng.choice(dv, 2, replace=False)
                if rng.random() < 0.33:
                    x = int(rng.integers(0, 2))
                    if y == x:
                        y = 2
                if rng.random() < self_loop_rate:
                    y = x
            out.append((a, b, int(x), int(y)))
        return out

    init = np.unique(_sym_keys(orc, rand_pairs(2500, dv0)))
    eng.build_index(init, dv0)
    orc.build(init, dv0)
    dv = dv0
    for b in range(6):
        dv += int(rng.integers(0, 8))
        ins = _sym_keys(orc, rand_pairs(int(rng.integers(0, 80)), dv))
        cur = orc.dump()
        dele = cur[rng.choice(len(cur), min(len(cur), int(rng.integers(0, 60))), replace=False)] if len(cur) else cur
        # removing a key also removes its mirror, keeping the lists symmetric
        rev = []
        for k in dele:
            d = int(k >> np.uint64(59)); u = int((k >> np.uint64(32)) & np.uint64(0x7FFFFFF)); v = int(k & np.uint64(0xFFFFFFFF))
            src = [s for s in range(qv) for t in range(qv) if orc.L.orc_dir(orc.h, s, t) == d][0]
            dst = [t for t in range(qv) if orc.L.orc_dir(orc.h, src, t) == d][0]
            rev.append(_key(orc.L.orc_dir(orc.h, dst, src), v, u))
        dele = np.concatenate([dele, np.array(rev, dtype=np.uint64)]) if len(rev) else dele
        delta_pairs = rand_pairs(int(rng.integers(0, 40)), dv)
        # a batch's delta edges are distinct (the input contract; the reference
        # double counts a repeated edge, and a counted tail cannot follow that)
        delta = np.unique(_sym_keys(orc, delta_pairs))
        # delta keys are also removed from the old index (ConstructUpdate, calig.cpp:776-804)
        dele = np.concatenate([dele, delta]).astype(np.uint64)
        c = eng.apply_batch(dv, ins, dele, delta)
        co = orc.batch(dv, ins, dele, delta, None, bind.PER_EDGE)
        assert c == co, f"seed {seed} batch {b}: engine {c} != oracle {co}"
        assert np.array_equal(eng.edge_counts(), orc.edge_counts())
        assert np.array_equal(eng.read_index(), orc.dump())
    eng.close()


def test_edge_cases():
    qedges = [(0, 1), (1, 2), (0, 2)]
    eng = Engine()
    eng.load_query(3, qedges)
    orc = bind.Oracle(3, qedges)
    d01, d10 = eng.query_dir(0, 1), eng.query_dir(1, 0)
    assert d01 == orc.L.orc_dir(orc.h, 0, 1) and d10 == orc.L.orc_dir(orc.h, 1, 0)
    # empty initial index
    eng.build_index(np.zeros(0, np.uint64), 4)
    orc.build(np.zeros(0, np.uint64), 4)
    assert len(eng.read_index()) == 0
    # empty batch
    assert eng.apply_batch(4, np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0, np.uint64)) == 0
    # triangle 0-1-2 fully in delta: counted once per query edge? only via the max edge
    tri = []
    for (a, b), (x, y) in zip(qedges, [(0, 1), (1, 2), (0, 2)]):
        tri += [_key(eng.query_dir(a, b), x, y), _key(eng.query_dir(b, a), y, x)]
    tri = np.array(tri, dtype=np.uint64)
    dup_ins = np.concatenate([tri[:2], tri[:2]])  # duplicate inserts are deduplicated
    c = eng.apply_batch(5, dup_ins, tri, tri)  # dv grows 4 -> 5
    co = orc.batch(5, dup_ins, tri, tri, None, bind.PER_EDGE)
    assert c == co
    assert np.array_equal(eng.read_index(), orc.dump())
    # removing keys that are absent is a no-op; delta empty -> no matching, no merge-back
    absent = np.array([_key(d01, 3, 4)], dtype=np.uint64)
    assert eng.apply_batch(5, np.zeros(0, np.uint64), absent, np.zeros(0, np.uint64)) == 0
    orc.batch(5, np.zeros(0, np.uint64), absent, np.zeros(0, np.uint64), None, bind.PER_EDGE)
    assert np.array_equal(eng.read_index(), orc.dump())
    # out-of-range keys are rejected with ERR_ARG and leave the handle usable
    bad = np.array([_key(d01, 7, 1)], dtype=np.uint64)
    with pytest.raises(CgbError):
        eng.apply_batch(5, bad, np.zeros(0, np.uint64), np.zeros(0, np.uint64))
    # decreasing dv_count is rejected
    with pytest.raises(CgbError):
        eng.apply_batch(4, np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0, np.uint64))
    eng.close()


@pytest.mark.parametrize("name", ["t_er5", "t_er_sparse"])
def test_cli_drop_in_total(name, workdir):
    """The drop-in CLI prints the reference's `Num Positive Matches` total."""
    import os
    import re
    import subprocess

    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cgbdsm_b200", "cgbdsm")
    out = subprocess.run([exe, p["query"], p["data"], p["update"], "0", str(spec.cli_batch_size)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    got = int(re.search(r"Num Positive Matches: (\d+)", out.stdout).group(1))
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    while ref.step() >= 0:
        pass
    assert got == ref.L.cgbref_total_count(ref.h)
    ref.close()


@pytest.mark.parametrize("name", ["t_er_sparse", "t_rmat"])
def test_seed_shards_sum_to_full_count(name, workdir):
    """Multi-GPU split: shards (run one after another on one GPU) add up to the
    unsharded count of every batch, and every shard keeps the full index."""
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    ref.set_count(False)
    ql, qe = read_query(p["query"])
    init = ref.init_keys()
    engines = [Engine(shard_index=i, num_shards=3) for i in range(3)]
    full = Engine()
    for e in engines + [full]:
        e.load_query(len(ql), qe, ql)
        e.build_index(init, ref.dv_count)
    while ref.step() >= 0:
        r = ref.last()
        args = (r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
        parts = [e.apply_batch(*args) for e in engines]
        assert sum(parts) == full.apply_batch(*args)
    idx = full.read_index()
    for e in engines:
        assert np.array_equal(e.read_index(), idx)
        e.close()
    full.close()
    ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["t_tiny", "t_er5", "t_er_sparse", "t_er_tree", "t_rmat"])
def test_valid_bits_match_restatement(name, workdir):
    """Valid bits (BuildLocalIndexBitAll) equal the restatement's word for word
    after every matched batch; the starting edge equals the reference
    planner's; pruning the matcher by them leaves every count unchanged."""
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    ql, qe = read_query(p["query"])
    o = bind.Oracle(len(ql), qe)
    go = ref.global_order()
    start = o.starting_edge(ref.cardinalities(), ref.avg_degrees())
    o.set_valid_bits(1, start)
    init = ref.init_keys()
    o.build(init, ref.dv_count)
    engs = []
    for flags in (FLAG_VALID_BITS, FLAG_MASK_PRUNE):
        e = Engine(flags=flags)
        e.load_query(len(ql), qe, ql)
        e.build_index(init, ref.dv_count)
        assert e.starting_edge() == start == (int(go[0]), int(go[1]))
        engs.append(e)
    matched = 0
    while ref.step() >= 0:
        r = ref.last()
        co = o.batch(r["dv"], r["ins"], r["del"], r["delta"], None, bind.PER_EDGE)
        for e in engs:
            assert e.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"]) == r["count"] == co
        if len(r["delta"]):
            matched += 1
            want = o.valid_bits()
            for e in engs:
                got, ms = e.valid_bits()
                assert np.array_equal(got, want), f"{name}: valid bits differ"
    assert matched > 0
    ref.close()


@pytest.mark.parametrize("name", ["c2", "c3_sparse"])
def test_index_symmetric_on_full_streams(name, workdir):
    """The matcher seeds each query edge from its own delta entries; that gives
    the reference's counts when every index list has its mirror ((a -> b)
    holds y at x iff (b -> a) holds x at y).  Checked on the device after
    every batch of the full R-MAT 1M/10M stream (9-vertex dense pattern) and
    of the R-MAT 4M/34M stream (7-vertex sparse pattern), with the product's
    producer making the keys."""
    from cgbdsm_b200 import Producer

    spec = SPECS[name]
    p = materialize(spec, workdir)
    ql, qe = read_query(p["query"])
    prod = Producer(p["query"], p["data"], p["update"], spec.cli_batch_size)
    init, dv = prod.initial()
    eng = Engine(dfs_budget_ms=120000)
    eng.load_query(len(ql), qe, ql)
    eng.build_index(init, dv)
    assert eng.check_symmetry() == 0
    for b in range(prod.num_batches):
        r = prod.next()
        eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
        assert eng.check_symmetry() == 0, f"{name} batch {b}: index lists not symmetric"
    eng.close()
    prod.close()


def test_check_symmetry_sees_a_missing_mirror():
    """The symmetry check counts an entry whose mirror is absent."""
    qedges = [(0, 1), (1, 2)]
    eng = Engine()
    eng.load_query(3, qedges)
    d01, d10 = eng.query_dir(0, 1), eng.query_dir(1, 0)
    keys = np.array([_key(d01, 1, 2), _key(d10, 2, 1), _key(d01, 3, 4)], dtype=np.uint64)
    eng.build_index(keys, 8)
    assert eng.check_symmetry() == 1
    eng.close()


@pytest.mark.parametrize("name", ["c2"])
def test_seed_shards_match_counted_tail_restatement(name, workdir):
    """The benchmark pattern's counts (~10^16 per batch) cannot be enumerated
    on a CPU; shards of its seed groups can be counted by the oracle's
    independent counted-tail restatement (inclusion-exclusion over set
    partitions of the tail, pinned to the reference's CPU path).  The engine,
    restricted to the same shards (same hash of (query edge, vertex at the
    plan's first position)), must give the same count and the same per-edge
    counts, bit for bit (tests/golden/shards_<name>.json)."""
    import json
    import os

    from cgbdsm_b200 import Producer

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"shards_{name}.json")
    g = json.load(open(path))
    spec = SPECS[name]
    assert g["spec"] == repr(spec)
    p = materialize(spec, workdir)
    ql, qe = read_query(p["query"])
    prod = Producer(p["query"], p["data"], p["update"], spec.cli_batch_size)
    init, dv = prod.initial()
    nb = max(len(s["batches"]) for s in g["shards"])
    batches = [prod.next() for _ in range(nb)]
    prod.close()
    for sh in g["shards"]:
        eng = Engine(shard_index=sh["shard"], num_shards=g["num_shards"], dfs_budget_ms=120000)
        eng.load_query(len(ql), qe, ql)
        eng.build_index(init, dv)
        assert [eng.plan_anchor(e) for e in range(len(qe))] == g["anchors"]
        for want in sh["batches"]:
            r = batches[want["batch"]]
            c = eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
            assert c == want["count"], f"shard {sh['shard']} batch {want['batch']}: {c} != {want['count']}"
            assert [int(x) for x in eng.edge_counts()] == want["edge_counts"]
        eng.close()


def test_c2_patterns_match_reference_at_full_size(workdir, tmp_path):
    """Patterns on the full R-MAT 1M/10M stream (batches of 100,000) whose
    counts the reference's enumerating CPU path can reach: its counts
    (tests/golden/c2_patterns.json, made by make_c2_golden.py from
    oracle/_ref) equal the plain pipeline's (product producer + engine) and
    the multi-query engine's, batch by batch."""
    import json
    import os

    from cgbdsm_b200 import MultiQuery, Producer
    from cgbdsm_b200.workloads import GraphData

    g_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_patterns.json")
    gold = json.load(open(g_path))
    spec = SPECS["c2"]
    assert gold["spec"] == repr(spec)
    p = materialize(spec, workdir)
    g = GraphData(spec)
    m = MultiQuery(dfs_budget_ms=120000)
    m.load_graph(g.labels, g.initial)
    ids = [m.register(len(q["labels"]), [tuple(e) for e in q["edges"]], q["labels"]) for q in gold["patterns"]]
    nb = max(len(q["reference_counts"]) for q in gold["patterns"])
    mq = []
    for b, batch in enumerate(g.batches()[:nb]):
        pos, _ = m.apply_batch(ins=batch)
        mq.append([int(pos[i]) for i in ids])
    m.close()
    for k, q in enumerate(gold["patterns"]):
        want = q["reference_counts"]
        assert [mq[b][k] for b in range(len(want))] == want, f"pattern {q['index']}: multi-query"
        qp = str(tmp_path / f"q{k}.graph")
        with open(qp, "w") as f:
            for i, lb in enumerate(q["labels"]):
                f.write(f"v {i} {lb}\n")
            for a, b in q["edges"]:
                f.write(f"e {a} {b} 0\n")
        prod = Producer(qp, p["data"], p["update"], spec.cli_batch_size)
        init, dv = prod.initial()
        eng = Engine(dfs_budget_ms=120000)
        eng.load_query(len(q["labels"]), [tuple(e) for e in q["edges"]], q["labels"])
        eng.build_index(init, dv)
        got = []
        for _ in want:
            r = prod.next()
            got.append(eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"]))
        eng.close()
        prod.close()
        assert got == want, f"pattern {q['index']}: plain pipeline"


@pytest.mark.gpu
def test_two_live_engines_keep_their_own_plans(workdir):
    """Two handles in one process (different patterns, both indexes built
    before either matches, batches interleaved): each engine's counts equal
    the reference's for its own pattern.  Plans and valid-bit plans are per
    handle, so building the second engine leaves the first one's intact.
    (The reference's CPU library keeps global state, so its two runs are
    recorded one after the other first.)"""
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    names = ["t_er_tree", "t_er_sparse"]
    runs, engs = [], []
    for name in names:
        spec = SPECS[name]
        p = materialize(spec, workdir)
        ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
        run = {"init": ref.init_keys(), "dv": ref.dv_count, "batches": []}
        while ref.step() >= 0:
            run["batches"].append(ref.last())
        ref.close()
        runs.append(run)
        qlabels, qedges = read_query(p["query"])
        e = Engine(flags=FLAG_MASK_PRUNE)  # the valid-bit plans steer the pruning
        e.load_query(len(qlabels), qedges, qlabels)
        engs.append(e)
    for run, e in zip(runs, engs):
        e.build_index(run["init"], run["dv"])
    for b in range(max(len(r["batches"]) for r in runs)):
        for k, (run, e) in enumerate(zip(runs, engs)):
            if b < len(run["batches"]):
                r = run["batches"][b]
                c = e.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
                assert c == r["count"], f"{names[k]} batch {b}: engine {c} != reference {r['count']}"
    for e in engs:
        e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,dense", [("t_er_tree_u", True), ("t_er_tree_s", False), ("t_rmat_tree", None)])
def test_level_sum_workloads_reach_their_plans(name, dense, workdir):
    """The level-sum parity workloads plan the counting they are there to
    test (their counts are checked against the reference with and without
    level sums by test_engine_matches_reference_cpu_path): every query label
    distinct gives sums over several positions, precomputed per vertex; a
    label shared with prefix positions gives the one-position sums with
    prefix vertices subtracted."""
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    spec = SPECS[name]
    p = materialize(spec, workdir)
    qlabels, qedges = read_query(p["query"])
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    eng = Engine()
    eng.load_query(len(qlabels), qedges, qlabels)
    eng.build_index(ref.init_keys(), ref.dv_count)
    ref.close()
    info = [eng.plan_info(ei) for ei in range(len(qedges))]
    eng.close()
    summed = [x for x in info if x["sum_from"]]
    assert summed, info
    if dense is True:
        assert any(x["dense"] and x["sum_from"] + 1 < x["n_core"] for x in summed), info
    elif dense is False:
        assert any(not x["dense"] and x["sum_from"] + 1 == x["n_core"] for x in summed), info


# the 7-vertex sparse pattern of the R-MAT 4M/34M benchmark (labels, edges)
C3_SPARSE_PATTERN = ([7, 6, 2, 0, 19, 10, 6], [(0, 1), (0, 2), (1, 3), (1, 4), (1, 5), (1, 6), (5, 6)])


@pytest.mark.gpu
def test_memoized_subtrees_match_reference(workdir, tmp_path):
    """The benchmark's sparse pattern on a small graph with its label
    distribution: one edge plan counts the subtree below the hub vertex once
    per (plan, vertex) and launch (EdgePlan.memo_from).  Counts equal the
    reference's CPU path with memos and level sums on and off, in the
    single-query and the multi-query engine."""
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    from cgbdsm_b200 import MultiQuery
    from cgbdsm_b200.workloads import GraphData

    spec = SPECS["t_rmat32"]
    p = materialize(spec, workdir)
    labels, edges = C3_SPARSE_PATTERN
    qp = str(tmp_path / "sparse.graph")
    with open(qp, "w") as f:
        for i, lb in enumerate(labels):
            f.write(f"v {i} {lb}\n")
        for a, b in edges:
            f.write(f"e {a} {b} 0\n")
    ref = bind.RefPipeline(qp, p["data"], p["update"], spec.cli_batch_size)
    init, dv = ref.init_keys(), ref.dv_count
    batches = []
    while ref.step() >= 0:
        batches.append(ref.last())
    ref.close()
    want = [r["count"] for r in batches]
    assert sum(want) > 0
    for flags in (0, FLAG_NO_LEVEL_SUM):
        eng = Engine(flags=flags)
        eng.load_query(len(labels), edges, labels)
        eng.build_index(init, dv)
        memo = [eng.plan_info(ei)["memo_from"] for ei in range(len(edges))]
        assert (any(memo) if flags == 0 else not any(memo)), memo
        got = [eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"]) for r in batches]
        eng.close()
        assert got == want, f"flags {flags}"
    g = GraphData(spec)
    m = MultiQuery(dfs_budget_ms=120000)
    m.load_graph(g.labels, g.initial)
    qid = m.register(len(labels), edges, labels)
    got = [int(m.apply_batch(ins=b)[0][qid]) for b in g.batches()]
    m.close()
    assert got == want, "multi-query engine"


@pytest.mark.gpu
@pytest.mark.parametrize("lane_max", [0, 2])
def test_pair_counting_mixed_with_descent(lane_max, workdir, tmp_path, monkeypatch):
    """Pair counting at the last core position (EdgePlan.pair_last) counts
    the candidates whose shorter list is at most $CGB_PAIR_LANE_MAX entries
    per lane and lets the others descend; shared work from that depth must
    not count a chunk's candidates twice.  With the bound at 0 or 2 every
    chunk mixes both kinds, and every chunk is shared (FLAG_FORCE_SPLIT):
    counts equal the reference's on C1 and on the benchmark's sparse
    pattern (single-query and multi-query engine)."""
    if not bind.have_ref():
        pytest.skip("oracle/_ref/libcgbref.so not built")
    from cgbdsm_b200 import MultiQuery
    from cgbdsm_b200.workloads import GraphData

    monkeypatch.setenv("CGB_PAIR_LANE_MAX", str(lane_max))
    labels, edges = C3_SPARSE_PATTERN
    qp = str(tmp_path / "sparse.graph")
    with open(qp, "w") as f:
        for i, lb in enumerate(labels):
            f.write(f"v {i} {lb}\n")
        for a, b in edges:
            f.write(f"e {a} {b} 0\n")
    for name, query in [("c1", None), ("t_rmat32", qp)]:
        spec = SPECS[name]
        p = materialize(spec, workdir)
        qfile = query or p["query"]
        ref = bind.RefPipeline(qfile, p["data"], p["update"], spec.cli_batch_size)
        init, dv = ref.init_keys(), ref.dv_count
        batches = []
        while ref.step() >= 0:
            batches.append(ref.last())
        ref.close()
        ql, qe = read_query(qfile)
        eng = Engine(flags=FLAG_FORCE_SPLIT)
        eng.load_query(len(ql), qe, ql)
        eng.build_index(init, dv)
        assert any(eng.plan_info(ei)["n_core"] >= 4 for ei in range(len(qe)))
        got = [eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"]) for r in batches]
        eng.close()
        assert got == [r["count"] for r in batches], name
        if query:
            g = GraphData(spec)
            m = MultiQuery(dfs_budget_ms=120000)
            m.load_graph(g.labels, g.initial)
            qid = m.register(len(ql), qe, ql)
            got = [int(m.apply_batch(ins=b)[0][qid]) for b in g.batches()]
            m.close()
            assert got == [r["count"] for r in batches], "multi-query engine"
