"""Serving loop (cgb_server_*, through the C ABI): requests submitted from a
client thread while earlier ones run on the device; each query's result for
each batch equals its result alone (the multi-query engine holding only that
query, on the same batch sequence), whichever queries were registered
around it."""
import numpy as np
import pytest

from cgbdsm_b200 import MultiQuery, Server
from cgbdsm_b200.engine import MQ_FLAG_NO_AUTOTUNE
from cgbdsm_b200.serve import cut_batches, run_schedule
from cgbdsm_b200.workloads import SPECS, GraphData

pytestmark = pytest.mark.gpu


def _queries(g, n, seed0):
    out = []
    for i in range(n):
        q = g.query([0, 1, 2][i % 3], 4 + i % 3, seed0 + i, 16)
        if q is not None:
            out.append(q)
    return out


def _alone(g, q, batches):
    m = MultiQuery(flags=MQ_FLAG_NO_AUTOTUNE, dfs_budget_ms=60000)
    m.load_graph(g.labels, g.initial)
    qid = m.register(len(q[0]), q[1], q[0])
    out = []
    for b in batches:
        pos, _ = m.apply_batch(ins=b)
        out.append(int(pos[qid]))
    m.close()
    return out


@pytest.mark.parametrize("staging", [1 << 20, 64 << 20])
def test_each_result_same_alone_and_in_the_mix(staging):
    """Batches of log-uniform sizes arrive every 0-3 ms, queries register in
    between; a 1 MiB staging ring makes later batches wait for space (they
    are admitted as earlier ones complete)."""
    g = GraphData(SPECS["t_rmat"])
    batches = cut_batches(g.stream, seed=7, lo=20, hi=2000, limit=14)
    qs = _queries(g, 6, 300)
    rng = np.random.default_rng(9)
    events, t = [], 0.0
    reg_at = {0: 0, 1: 0, 2: 4, 3: 7, 4: 7, 5: 10}  # query -> number of batches submitted before it
    for i, b in enumerate(batches):
        for k, at in reg_at.items():
            if at == i and k < len(qs):
                events.append((t, "register", qs[k]))
        t += float(rng.uniform(0, 0.003))
        events.append((t, "batch", b))
    srv = Server(g.labels, g.initial, staging_bytes=staging, dfs_budget_ms=60000)
    res = run_schedule(srv, events)
    srv.close()
    qid_of, live, per_batch = {}, [], []
    k_reg = 0
    for r in res:
        assert r["status"] == 0, r
        if r["what"] == "register":
            qid_of[k_reg] = r["query_id"]
            live.append(k_reg)
            k_reg += 1
        else:
            per_batch.append((list(live), r["pos"].copy()))
    assert len(per_batch) == len(batches)
    for k, q in enumerate(qs):
        want = _alone(g, q, batches)
        got = [int(pos[qid_of[k]]) for lv, pos in per_batch if k in lv]
        first = reg_at[k]
        assert got == want[first:], f"query {k}"
    assert any(int(pos.sum()) for _, pos in per_batch)


def test_deletion_batches_and_oversize_rejection():
    """A deletion batch through the server returns negative matches equal to
    the engine's; a batch larger than the staging ring is rejected with
    CGB_ERR_LIMIT and the requests after it still run."""
    g = GraphData(SPECS["t_rmat"])
    q = _queries(g, 1, 400)[0]
    srv = Server(g.labels, g.initial, staging_bytes=1 << 20)
    srv.wait(srv.submit_register(len(q[0]), q[1], q[0]))
    b0, b1 = g.stream[:500], g.stream[500:900]
    big = np.tile(g.stream[:100], (2000, 1))  # 200,000 pairs = 1.6 MB > ring
    t = [srv.submit_batch(ins=b0), srv.submit_batch(ins=big), srv.submit_batch(ins=b1),
         srv.submit_batch(dele=b0[:200])]
    r = [srv.wait(x) for x in t]
    srv.close()
    assert r[1]["status"] == 4
    assert r[0]["status"] == r[2]["status"] == r[3]["status"] == 0
    m = MultiQuery(flags=MQ_FLAG_NO_AUTOTUNE)
    m.load_graph(g.labels, g.initial)
    qid = m.register(len(q[0]), q[1], q[0])
    p0, _ = m.apply_batch(ins=b0)
    p1, _ = m.apply_batch(ins=b1)
    _, n3 = m.apply_batch(dele=b0[:200])
    m.close()
    assert int(r[0]["pos"][0]) == int(p0[qid])
    assert int(r[2]["pos"][0]) == int(p1[qid])
    assert int(r[3]["neg"][0]) == int(n3[qid])
