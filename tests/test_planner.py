"""Matching plans (cgbdsm_b200/csrc/query.cpp, plan_edges) against the
conditions that make their counting shortcuts exact, on the headline's
patterns, the 64- and 16-query sets and the parity workloads' patterns.  The
GPU parity tests check the counts; these check, without a GPU, that every
plan which takes a shortcut satisfies the conditions it relies on:

  level sums over several positions (dense): one backward list per position,
      labels of their own for the positions and their pendant tails
  one-position level sums: one backward list at the last core position, its
      pendants exclude no prefix vertex, no other tail shares its label
  subtree memos: every list below the split hangs off the key position or
      the range, and the range's labels meet no other prefix position
  per-lane pendant tails: tails off the last core vertex have one list and a
      label group of their own
  pair counting: the last core position has two lists, one owned by the
      position before it, and no tail list or exclusion involves either
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
from collections import Counter

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cgbdsm_b200", "csrc")

C3_TREE = ([0, 23, 25, 6, 14, 2, 1], [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6)])
C3_SPARSE = ([7, 6, 2, 0, 19, 10, 6], [(0, 1), (0, 2), (1, 3), (1, 4), (1, 5), (1, 6), (5, 6)])


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("planner")
    exe = str(d / "plan_dump")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                    os.path.join(ROOT, "tests", "native", "plan_dump.cpp"), os.path.join(CSRC, "query.cpp"),
                    "-o", exe], check=True)
    counter = [0]

    def run(labels, edges, mq=False):
        counter[0] += 1
        qp = str(d / f"q{counter[0]}.graph")
        with open(qp, "w") as f:
            for i, lb in enumerate(labels):
                f.write(f"v {i} {lb}\n")
            for a, b in edges:
                f.write(f"e {a} {b} 0\n")
        out = subprocess.run([exe, qp] + (["mq"] if mq else []), capture_output=True, text=True, check=True).stdout
        plans = []
        for line in out.splitlines():
            head, vs, off, pos, excl, gid = line.split("|")
            f = [int(x) for x in head.split()]
            plans.append({"ei": f[0], "n": f[1], "nc": f[2], "sum_from": f[3], "dense": f[4], "sum_tails": f[5],
                          "sum_same": f[6], "memo_from": f[7], "memo_pos": f[8], "grouped": f[9], "hit_mask": f[10],
                          "tail_lane": f[11], "pair_last": f[12], "pair_a": f[13], "pair_b": f[14],
                          "pair_excl": f[15], "vs": [int(x) for x in vs.split()],
                          "off": [int(x) for x in off.split()], "pos": [int(x) for x in pos.split()],
                          "excl": [int(x) for x in excl.split()], "gid": [int(x) for x in gid.split()]})
        return plans
    return run


def _lists(p, t):
    return p["pos"][p["off"][t]:p["off"][t + 1]]


def _alone(p, t):
    g = p["gid"]
    return (t == p["nc"] or g[t - 1] != g[t]) and (t + 1 == p["n"] or g[t + 1] != g[t])


def check_plan(p, labels):
    nc, n, vs = p["nc"], p["n"], p["vs"]
    lab = [labels[v] for v in vs]
    count = Counter(labels)
    assert sorted(vs) == list(range(n))
    for k in range(2, n):  # every later position has a backward neighbour
        assert len(_lists(p, k)) >= 1 and all(x < k and x < nc for x in _lists(p, k))
    if p["tail_lane"] == 2:
        for t in range(nc, n):
            if nc - 1 in _lists(p, t):
                assert len(_lists(p, t)) == 1 and _alone(p, t)
    s = p["sum_from"]
    if s and p["dense"]:
        assert 2 <= s and s + 1 < nc and p["sum_same"] == 0
        for k in range(s, nc):
            assert len(_lists(p, k)) == 1 and count[lab[k]] == 1
            for t in range(nc, n):
                if k in _lists(p, t):
                    assert _lists(p, t) == [k] and _alone(p, t) and count[lab[t]] == 1
                    assert (p["sum_tails"] >> t) & 1
    elif s:
        j = nc - 1
        assert s == j and len(_lists(p, j)) == 1
        assert not (p["grouped"] and (p["hit_mask"] >> j) & 1)
        for t in range(nc, n):
            if j in _lists(p, t):
                assert (p["excl"][t] & ((1 << j) - 1)) == 0
            else:
                assert not (p["excl"][t] >> j) & 1
        assert p["sum_same"] == sum(1 << t for t in range(j) if lab[t] == lab[j])
    m, key = p["memo_from"], p["memo_pos"]
    if m:
        assert key < m and m + 2 <= nc
        assert not (p["grouped"] and key < 2)
        inside = lambda x: x == key or x >= m  # noqa: E731
        for k in range(m, nc):
            assert all(inside(x) for x in _lists(p, k))
            assert all(lab[k] != lab[c] for c in range(m) if c != key)
        for t in range(nc, n):
            assert all(inside(x) for x in _lists(p, t))
            assert all(not (p["excl"][t] >> c) & 1 for c in range(m) if c != key)
        if p["grouped"]:
            assert p["hit_mask"] >> m == 0
        assert not (p["dense"] and s <= m)
    if p["pair_last"]:
        j = nc - 1
        lists = list(range(p["off"][j], p["off"][j + 1]))
        assert len(lists) == 2 and sorted([p["pair_a"], p["pair_b"]]) == lists
        assert p["pos"][p["pair_b"]] == j - 1 and p["pos"][p["pair_a"]] < j - 1
        for t in range(nc, n):
            assert all(x < j - 1 for x in _lists(p, t)) and ((p["excl"][t] >> (j - 1)) & 3) == 0
        if p["grouped"]:
            assert ((p["hit_mask"] >> (j - 1)) & 3) == 0
        assert p["pair_excl"] == sum(1 << t for t in range(j - 1) if lab[t] == lab[j])


def test_headline_patterns_plan_their_shortcuts(dump):
    tree = dump(*C3_TREE)
    assert all(p["dense"] and p["sum_from"] == 2 for p in tree)
    sparse = dump(*C3_SPARSE)
    memo = [(p["ei"], p["memo_from"], p["memo_pos"]) for p in sparse if p["memo_from"]]
    assert memo == [(1, 3, 2)]  # edge (0, 2): the subtree below the hub vertex 1
    assert sparse[1]["pair_last"]  # and its last level is one intersection per lane
    for labels, edges, plans in [(*C3_TREE, tree), (*C3_SPARSE, sparse)]:
        for p in plans:
            check_plan(p, labels)
    # the multi-query engine plans no dense sums
    assert not any(p["dense"] for p in dump(*C3_TREE, mq=True))


@pytest.mark.parametrize("qset", ["c2", "c3"])
def test_query_set_plans_meet_their_conditions(dump, qset):
    qs = json.load(open(os.path.join(ROOT, "cgbdsm_b200", "data", f"queries_{qset}.json")))["queries"]
    seen = Counter()
    for q in qs:
        edges = [tuple(e) for e in q["edges"]]
        for mq in (False, True):
            if not mq and len(edges) > 16:
                continue
            for p in dump(q["labels"], edges, mq=mq):
                check_plan(p, q["labels"])
                seen["dense"] += p["dense"]
                seen["one"] += bool(p["sum_from"]) and not p["dense"]
                seen["memo"] += bool(p["memo_from"])
                seen["pair"] += p["pair_last"]
    assert seen["one"] > 0, seen


def test_parity_workload_plans_meet_their_conditions(dump, tmp_path):
    from cgbdsm_b200.workloads import SPECS, materialize, read_query

    for name in ["t_tiny", "t_er5", "t_er6", "t_er_sparse", "t_er_tree", "t_rmat", "c1", "c1_q25", "t_er_tree_u",
                 "t_er_tree_s", "t_rmat_tree"]:
        paths = materialize(SPECS[name], str(tmp_path))
        labels, edges = read_query(paths["query"])
        for p in dump(labels, edges):
            check_plan(p, labels)
