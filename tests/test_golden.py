"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the
reference's own CPU path) replayed without the reference tree:

  * the seeded generator still writes the inputs the fixtures were made from,
  * the restatement (oracle/oracle.c) replays t_tiny from the stored keys,
  * the product's producer emits the reference's key multisets, and the
    restatement on those keys gives the reference's counts and final index,
  * (GPU) the engine on the producer's keys gives the same counts and index,

for the text inputs and for the reference's binary CSR input path (<name>_csr).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from cgbdsm_b200 import Producer
from cgbdsm_b200.workloads import SPECS, materialize, read_query, write_binary_csr
from oracle import bind

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["t_tiny", "t_er5", "t_er_tree", "t_er_sparse", "t_rmat", "c1", "c1_q25"]
BINARY = ["t_er5_csr", "t_rmat_csr"]


def load(name):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        return json.load(f)


def to_original(keys, new2old):
    n2o = new2old.astype(np.uint64)
    d = keys >> np.uint64(59)
    u = (keys >> np.uint64(32)) & np.uint64(0x7FFFFFF)
    v = keys & np.uint64(0xFFFFFFFF)
    return np.sort((d << np.uint64(59)) | (n2o[u] << np.uint64(32)) | n2o[v])


def digest(keys):
    a = np.ascontiguousarray(np.sort(keys).astype("<u8"))
    return [int(a.size), hashlib.sha256(a.tobytes()).hexdigest()]


@pytest.mark.parametrize("name", NAMES)
def test_generator_reproduces_golden_inputs(name, workdir):
    g = load(name)
    assert g["spec"] == repr(SPECS[name]), "workload spec changed since the fixture was made"
    p = materialize(SPECS[name], workdir)
    for k, h in g["inputs"].items():
        assert hashlib.sha256(open(p[k], "rb").read()).hexdigest() == h, f"{name}: {k} input differs"


@pytest.mark.parametrize("name", BINARY)
def test_csr_writer_reproduces_golden_inputs(name, workdir):
    g = load(name)
    p = write_binary_csr(SPECS[g["workload"]], workdir, g["nvcls"])
    for suffix, h in g["inputs"].items():
        assert hashlib.sha256(open(p["data"] + suffix, "rb").read()).hexdigest() == h, f"{name}: {suffix} differs"


def _inputs(name, workdir):
    """(fixture, query, data, update) of a text or binary golden workload."""
    g = load(name)
    spec = SPECS[g["workload"]]
    if "nvcls" in g:
        p = write_binary_csr(spec, workdir, g["nvcls"])
        return g, spec, p["query"], p["data"], "-"
    p = materialize(spec, workdir)
    return g, spec, p["query"], p["data"], p["update"]


def test_restatement_replays_full_fixture():
    z = np.load(os.path.join(GOLDEN, "t_tiny_full.npz"))
    q = z["file_query"].tobytes().decode()
    labels, edges = {}, []
    for line in q.splitlines():
        t = line.split()
        if t and t[0] == "v":
            labels[int(t[1])] = int(t[2])
        elif t and t[0] == "e":
            edges.append((int(t[1]), int(t[2])))
    o = bind.Oracle(len(labels), edges)
    o.build(z["init"], int(z["dv0"]))
    b = 0
    while f"b{b}_meta" in z:
        dv, count = (int(x) for x in z[f"b{b}_meta"])
        got = o.batch(dv, z[f"b{b}_ins"], z[f"b{b}_del"], z[f"b{b}_delta"], None, bind.PER_EDGE)
        assert got == count, f"batch {b}: restatement {got} != reference {count}"
        b += 1
    assert b == load("t_tiny")["num_batches"]
    assert np.array_equal(to_original(o.dump(), z["new2old"]), z["final_original"])
    assert digest(z["final_original"]) == load("t_tiny")["final_index"]


def _producer_batches(name, workdir):
    """Runs the product's producer over the workload and checks every key
    multiset against the fixture; returns the batches for replay."""
    g, spec, query, data, update = _inputs(name, workdir)
    prod = Producer(query, data, update, spec.cli_batch_size)
    assert prod.num_batches == g["num_batches"]
    init, dv0 = prod.initial()
    assert dv0 == g["dv_initial"]
    assert digest(to_original(init, prod.new2old())) == g["initial_index"]
    batches = []
    for b, gb in enumerate(g["batches"]):
        r = prod.next()
        n2o = prod.new2old()
        assert r["dv"] == gb["dv"], f"batch {b}: dv"
        assert [int(x) for x in r["edge_ok"]] == gb["edge_ok"], f"batch {b}: edge_ok"
        assert digest(np.unique(to_original(r["ins"], n2o))) == gb["ins"], f"batch {b}: ins keys"
        assert digest(to_original(r["del"], n2o)) == gb["del"], f"batch {b}: del keys"
        assert digest(to_original(r["delta"], n2o)) == gb["delta"], f"batch {b}: delta keys"
        batches.append(r)
    n2o = prod.new2old()
    prod.close()
    ql, qe = read_query(query)
    return g, (init, dv0), batches, n2o, (ql, qe)


@pytest.mark.parametrize("name", NAMES + BINARY)
def test_producer_and_restatement_match_golden(name, workdir):
    g, (init, dv0), batches, n2o, (ql, qe) = _producer_batches(name, workdir)
    o = bind.Oracle(len(ql), qe)
    o.build(init, dv0)
    for b, (r, gb) in enumerate(zip(batches, g["batches"])):
        got = o.batch(r["dv"], r["ins"], r["del"], r["delta"], None, bind.PER_EDGE)
        assert got == gb["count"], f"{name} batch {b}: restatement {got} != reference {gb['count']}"
    assert digest(to_original(o.dump(), n2o)) == g["final_index"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES + BINARY)
def test_engine_matches_golden(name, workdir):
    from cgbdsm_b200 import Engine

    g, (init, dv0), batches, n2o, (ql, qe) = _producer_batches(name, workdir)
    eng = Engine(device=0)
    eng.load_query(len(ql), qe, ql)
    eng.build_index(init, dv0)
    for b, (r, gb) in enumerate(zip(batches, g["batches"])):
        got = eng.apply_batch(r["dv"], r["ins"], r["del"], r["delta"], r["edge_ok"])
        assert got == gb["count"], f"{name} batch {b}: engine {got} != reference {gb['count']}"
    assert digest(to_original(eng.read_index(), n2o)) == g["final_index"]
    eng.close()
