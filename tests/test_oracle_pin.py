"""Pins the C restatement (oracle/oracle.c) to the reference's own CPU path.

The reference has no tests or golden vectors of its own, so the restatement
is pinned by running the reference's unmodified CPU sources
(oracle/_ref/libcgbref.so: CaLiG, CPUIndexMirror, cpu_dfs) on the same
seeded workloads, and by an independent brute-force embedding count.
"""
import numpy as np
import pytest

from cgbdsm_b200.workloads import SPECS, materialize, read_query
from oracle import bind

PIN_CASES = ["t_tiny", "t_er5", "t_er6", "t_er_sparse", "t_er_tree", "c1", "c1_q25"]


def _ref_or_skip():
    if not bind.have_ref():
        pytest.skip("reference CPU path (oracle/_ref/libcgbref.so) not built")


def run_pin(name, workdir):
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    qlabels, qedges = read_query(p["query"])
    glob = bind.Oracle(len(qlabels), qedges)
    per = bind.Oracle(len(qlabels), qedges)
    tail = bind.Oracle(len(qlabels), qedges)
    init = ref.init_keys()
    glob.build(init, ref.dv_count)
    per.build(init, ref.dv_count)
    tail.build(init, ref.dv_count)
    go = ref.global_order()
    counts = []
    while True:
        b = ref.step()
        if b < 0:
            break
        r = ref.last()
        cg = glob.batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"], bind.GLOBAL, go)
        cp = per.batch(r["dv"], r["ins"], r["del"], r["delta"], None, bind.PER_EDGE)
        assert cg == r["count"], f"{name} batch {b}: global-order restatement {cg} != reference {r['count']}"
        assert cp == r["count"], f"{name} batch {b}: per-edge restatement {cp} != reference {r['count']}"
        ct = tail.batch(r["dv"], r["ins"], r["del"], r["delta"], None, bind.TAIL)
        assert ct == r["count"], f"{name} batch {b}: counted-tail restatement {ct} != reference {r['count']}"
        assert per.asymmetry() == 0, f"{name} batch {b}: index lists not symmetric"
        counts.append(cp)
    # index contents after the last merge-back, compared in original vertex ids
    n2o = ref.new2old().astype(np.uint64)
    mine = per.dump()
    d = mine >> np.uint64(59)
    u = (mine >> np.uint64(32)) & np.uint64(0x7FFFFFF)
    v = mine & np.uint64(0xFFFFFFFF)
    mine_orig = np.sort((d << np.uint64(59)) | (n2o[u] << np.uint64(32)) | n2o[v])
    assert np.array_equal(mine_orig, ref.dump_main_original_ids())
    ref.close()
    return spec, p, counts, (qlabels, qedges)


@pytest.mark.parametrize("name", PIN_CASES)
def test_restatement_matches_reference_cpu_path(name, workdir):
    _ref_or_skip()
    run_pin(name, workdir)


@pytest.mark.parametrize("name", ["t_tiny", "t_er5"])
def test_incremental_counts_equal_bruteforce_delta(name, workdir):
    """sum of batch counts == |Emb(Q, G_final)| - |Emb(Q, G_initial)| (insertion-only stream)."""
    _ref_or_skip()
    spec, p, counts, (ql, qe) = run_pin(name, workdir)
    n, glab, e0 = bind.read_graph(p["data"])
    upd = bind.read_updates(p["update"])
    o = bind.Oracle(len(ql), qe)
    before = o.bruteforce(n, e0, glab, ql, qe)
    after = o.bruteforce(n, np.concatenate([e0, upd]), glab, ql, qe)
    assert sum(counts) == after - before


@pytest.mark.parametrize("name", PIN_CASES + ["t_rmat"])
def test_valid_bit_plan_and_soundness(name, workdir):
    """The restated planner pieces the valid bits depend on (SelectStartingEdge,
    BuildIndexingOrder, rebuild flags; plan.cpp:428-533, 1180-1370) equal the
    reference planner's, and pruning the count with the restated valid bits
    leaves every batch count unchanged (they are a sound superset)."""
    _ref_or_skip()
    spec = SPECS[name]
    p = materialize(spec, workdir)
    ref = bind.RefPipeline(p["query"], p["data"], p["update"], spec.cli_batch_size)
    ql, qe = read_query(p["query"])
    o = bind.Oracle(len(ql), qe)
    go = ref.global_order()
    start = o.starting_edge(ref.cardinalities(), ref.avg_degrees())
    assert start == (int(go[0]), int(go[1]))
    qv = len(ql)
    for ei in range(len(qe)):
        rv, ro, rb = ref.indexing_order(ei)
        vs, offs, bni, vflags = o.indexing_order(ei, start)
        assert np.array_equal(rv, vs[:qv]) and np.array_equal(ro, offs[: qv + 1])
        assert np.array_equal(rb[1:], bni[1:])  # bni_[0] is a placeholder the reference never reads
        assert vflags == ref.rebuild_vertices(ei)
    plain, pruned = bind.Oracle(len(ql), qe), bind.Oracle(len(ql), qe)
    init = ref.init_keys()
    plain.build(init, ref.dv_count)
    pruned.build(init, ref.dv_count)
    pruned.set_valid_bits(2, start)
    while ref.step() >= 0:
        r = ref.last()
        c0 = plain.batch(r["dv"], r["ins"], r["del"], r["delta"], None, bind.PER_EDGE)
        c1 = pruned.batch(r["dv"], r["ins"], r["del"], r["delta"], None, bind.PER_EDGE)
        assert c0 == c1 == r["count"]
    ref.close()
