"""Packed-memory-array layout (cgb_gpma_*, the reference's GPMA rebuilt
without device-side launches): after a bulk load and after every batch
update, each direction's keys equal the set model (S + ins) - del, through
leaf windows, larger windows, deletions, re-insertions and rebuilds."""
import numpy as np
import pytest

from cgbdsm_b200 import Gpma

pytestmark = pytest.mark.gpu


def key(d, u, v):
    return (np.uint64(d) << np.uint64(59)) | (np.uint64(u) << np.uint64(32)) | np.uint64(v)


def rand_keys(rng, n, nd, nu, nv, hub_frac=0.0):
    d = rng.integers(0, nd, n).astype(np.uint64)
    u = rng.integers(0, nu, n).astype(np.uint64)
    if hub_frac:
        hub = rng.random(n) < hub_frac
        u[hub] = 7
    v = rng.integers(0, nv, n).astype(np.uint64)
    return (d << np.uint64(59)) | (u << np.uint64(32)) | v


def check(g, model, nd):
    low = np.uint64((1 << 59) - 1)
    for d in range(nd):
        want = np.array(sorted(k & low for k in model if int(k >> np.uint64(59)) == d), dtype=np.uint64)
        got = g.extract(d)
        assert np.array_equal(got, want), f"direction {d}: {len(got)} keys vs {len(want)}"


@pytest.mark.parametrize("seed", range(4))
def test_gpma_matches_set_model(seed):
    rng = np.random.default_rng(7000 + seed)
    nd = int(rng.integers(1, 6))
    nu, nv = 300, 5000
    g = Gpma(nd)
    init = rand_keys(rng, 20000, nd, nu, nv, hub_frac=0.2)
    g.bulk_load(np.concatenate([init, init[:500]]))  # duplicates allowed
    model = set(int(k) for k in init)
    model = set(np.uint64(k) for k in model)
    check(g, model, nd)
    rebuilt = 0
    for b in range(12):
        # growing batches force windows at every level and, eventually, rebuilds
        ins = rand_keys(rng, int(rng.integers(0, 4000 * (b + 1))), nd, nu, nv, hub_frac=0.3)
        cur = np.array(sorted(model), dtype=np.uint64)
        dele = cur[rng.choice(len(cur), min(len(cur), int(rng.integers(0, 3000))), replace=False)] if len(cur) else cur
        both = ins[: len(ins) // 10]  # keys both inserted and deleted: deleted
        dele = np.concatenate([dele, both, rand_keys(rng, 200, nd, nu, nv)])  # plus absent keys
        g.batch_update(ins, dele)
        model = (model | set(np.uint64(k) for k in ins)) - set(np.uint64(k) for k in dele)
        st = g.stats()
        rebuilt += st["rebuilt"]
        assert st["keys"] == len(model)
        check(g, model, nd)
    assert rebuilt >= 1, "the growing batches should have forced a rebuild"
    g.close()


def test_gpma_edge_cases():
    g = Gpma(3)
    g.bulk_load(np.zeros(0, np.uint64))
    for d in range(3):
        assert len(g.extract(d)) == 0
    g.batch_update(np.array([key(1, 2, 3)], np.uint64), np.zeros(0, np.uint64))
    assert list(g.extract(1)) == [(2 << 32) | 3]
    g.batch_update(np.zeros(0, np.uint64), np.array([key(1, 2, 3), key(0, 1, 1)], np.uint64))
    assert len(g.extract(1)) == 0
    # re-insert after delete, and a single hot row growing past several windows
    ks = np.array([key(2, 9, v) for v in range(5000)], np.uint64)
    for i in range(0, 5000, 500):
        g.batch_update(ks[i:i + 500], np.zeros(0, np.uint64))
    assert np.array_equal(g.extract(2), np.array([(9 << 32) | v for v in range(5000)], np.uint64))
    g.batch_update(ks[::2], ks[1::2])  # inserting present keys changes nothing
    assert np.array_equal(g.extract(2), np.array([(9 << 32) | v for v in range(0, 5000, 2)], np.uint64))
    with pytest.raises(Exception):
        g.batch_update(np.array([key(3, 0, 0)], np.uint64), np.zeros(0, np.uint64))  # direction 3 of 3
    g.close()
