"""The allocation-free index update (cgb_merge_keys_noalloc) against the engine.

Callers that cannot allocate device memory (code running under CUDA-graph
capture, hosts whose allocator owns every byte of device memory, plugins that
must not grow a process's footprint) get this entry point: it keeps all its
temporaries in a fixed static device array.  Here it is called through the C
ABI twice in a row (the second call reuses the scratch array after the first)
and its output is compared with the allocating path (cgb_build_index +
cgb_apply_batch + cgb_read_index) on the same edits: exact equality, as for
all integer results in this suite.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from cgbdsm_b200 import CgbError, Engine, engine

pytestmark = pytest.mark.gpu


def _key(d, u, v):
    return (np.uint64(d) << np.uint64(59)) | (np.uint64(u) << np.uint64(32)) | np.uint64(v)


def _engine_result(qv, qedges, old, dv, ins, dele):
    e = Engine()
    e.load_query(qv, qedges)
    e.build_index(old, dv)
    e.apply_batch(dv, ins, dele, np.zeros(0, np.uint64))
    out = e.read_index()
    e.close()
    return out


def _noalloc(lib, old, ins, dele, dv):
    import torch

    dev = torch.device("cuda", 0)
    t_old = torch.from_numpy(old.view(np.int64)).to(dev) if len(old) else torch.zeros(1, dtype=torch.int64, device=dev)
    t_ins = torch.from_numpy(ins.view(np.int64)).to(dev) if len(ins) else torch.zeros(1, dtype=torch.int64, device=dev)
    t_del = torch.from_numpy(dele.view(np.int64)).to(dev) if len(dele) else torch.zeros(1, dtype=torch.int64, device=dev)
    out = torch.zeros(max(1, len(old) + len(ins)), dtype=torch.int64, device=dev)
    n_out = torch.zeros(1, dtype=torch.int64, device=dev)
    st = lib.cgb_merge_keys_noalloc(t_old.data_ptr(), len(old), t_ins.data_ptr(), len(ins), t_del.data_ptr(),
                                    len(dele), dv, out.data_ptr(), n_out.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    n = int(n_out.item())
    return out[:n].cpu().numpy().view(np.uint64)


def test_noalloc_matches_engine_twice_in_a_row():
    lib = engine.load_library()
    rng = np.random.default_rng(7)
    qedges = [(0, 1), (1, 2), (0, 2), (2, 3)]
    nd, dv = 8, 5000
    old = np.unique(np.array([_key(rng.integers(0, nd), rng.integers(0, dv), rng.integers(0, dv))
                              for _ in range(60000)], dtype=np.uint64))
    state = old
    for call in range(2):
        ins = np.array([_key(rng.integers(0, nd), rng.integers(0, dv), rng.integers(0, dv))
                        for _ in range(20000)], dtype=np.uint64)
        ins = np.concatenate([ins, ins[:500]])  # duplicates are allowed
        dele = np.concatenate([state[rng.choice(len(state), 15000, replace=False)], ins[:300]])
        want = _engine_result(4, qedges, state, dv, ins, dele)
        got = _noalloc(lib, state, ins, dele, dv)
        assert np.array_equal(got, want), f"call {call}"
        state = got


def _noalloc_status(lib, old, ins, dele, dv):
    """Calls the entry point; returns (status, out_n as written by the device)."""
    import torch

    dev = torch.device("cuda", 0)
    t_old = torch.from_numpy(old.view(np.int64)).to(dev) if len(old) else torch.zeros(1, dtype=torch.int64, device=dev)
    t_ins = torch.from_numpy(ins.view(np.int64)).to(dev) if len(ins) else torch.zeros(1, dtype=torch.int64, device=dev)
    t_del = torch.from_numpy(dele.view(np.int64)).to(dev) if len(dele) else torch.zeros(1, dtype=torch.int64, device=dev)
    out = torch.zeros(max(1, len(old) + len(ins)), dtype=torch.int64, device=dev)
    n_out = torch.full((1,), 12345, dtype=torch.int64, device=dev)
    st = lib.cgb_merge_keys_noalloc(t_old.data_ptr(), len(old), t_ins.data_ptr(), len(ins), t_del.data_ptr(),
                                    len(dele), dv, out.data_ptr(), n_out.data_ptr(), None)
    torch.cuda.synchronize()
    return st, int(n_out.cpu().numpy().view(np.uint64)[0])


def test_noalloc_flags_keys_outside_the_vertex_range():
    """An edit key whose u or v is not below dv_count is not an error of the
    call (it returns CGB_OK, the check runs on the device) but makes the
    device write UINT64_MAX as the output length; the next call is unaffected."""
    lib = engine.load_library()
    dv = 100
    old = np.array([_key(0, 1, 2), _key(0, 1, 5), _key(1, 3, 4)], dtype=np.uint64)
    bad = np.array([_key(0, 1, 3), _key(0, 2, dv)], dtype=np.uint64)
    st, n = _noalloc_status(lib, old, bad, np.zeros(0, np.uint64), dv)
    assert st == 0 and n == 2**64 - 1
    absent = np.array([_key(0, 0, 0)], np.uint64)  # removing an absent key changes nothing
    st, n = _noalloc_status(lib, old, np.zeros(0, np.uint64), absent, dv)
    assert st == 0 and n == 3
    got = _noalloc(lib, old, bad[:1], old[1:2], dv)
    assert np.array_equal(got, np.sort(np.array([old[0], bad[0], old[2]], dtype=np.uint64)))


def test_noalloc_empty_inputs_and_many_tiles():
    """No old keys, no edits, and a merge that spans many 2048-entry tiles with
    long runs of equal (d, u) (a hub), each against the allocating path."""
    lib = engine.load_library()
    dv = 70000
    st, n = _noalloc_status(lib, np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0, np.uint64), dv)
    assert st == 0 and n == 0
    rng = np.random.default_rng(11)
    hub = np.array([_key(1, 7, v) for v in rng.choice(dv, 30000, replace=False)], dtype=np.uint64)
    rest = np.array([_key(rng.integers(0, 4), rng.integers(0, dv), rng.integers(0, dv)) for _ in range(20000)],
                    dtype=np.uint64)
    old = np.unique(np.concatenate([hub, rest]))
    ins = np.array([_key(1, 7, v) for v in rng.choice(dv, 20000, replace=False)], dtype=np.uint64)
    dele = old[rng.choice(len(old), 9000, replace=False)]
    want = _engine_result(3, [(0, 1), (1, 2)], old, dv, ins, dele)
    assert np.array_equal(_noalloc(lib, old, ins, dele, dv), want)
    assert np.array_equal(_noalloc(lib, np.zeros(0, np.uint64), ins, dele, dv), np.unique(np.setdiff1d(ins, dele)))


def test_noalloc_rejects_oversized_batches():
    lib = engine.load_library()
    too_many = engine.NOALLOC_MAX_EDITS + 1
    st = lib.cgb_merge_keys_noalloc(None, 0, ctypes.c_void_p(16), too_many, None, 0, 10, ctypes.c_void_p(16),
                                    ctypes.c_void_p(16), None)
    assert st == 4  # CGB_ERR_LIMIT, before any device work
