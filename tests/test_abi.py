"""The C-ABI library loads and exports every entry point include/cgbdsm.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

from cgbdsm_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "cgbdsm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cgb_[a-z_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(engine.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(engine.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_default_config_without_gpu():
    lib = engine.load_library()
    cfg = engine.Config(7, 1, 2, 3, 4, 5, 6)
    lib.cgb_default_config(ctypes.byref(cfg))
    assert (cfg.device, cfg.pool_words, cfg.dfs_blocks_per_sm, cfg.flags, cfg.dfs_budget_ms, cfg.shard_index,
            cfg.num_shards) == (0, 0, 0, 0, 0, 0, 0)


def test_noalloc_limits_checked_before_any_device_call():
    """The allocation-free index update refuses edit counts beyond its static scratch
    (CGB_ERR_LIMIT = 4) and missing pointers (CGB_ERR_ARG = 1) on the host, before any
    CUDA call, so these run without a GPU.  A pair of counts whose sum wraps 64 bits is
    refused too."""
    lib = engine.load_library()
    p = ctypes.c_void_p(16)
    cap = engine.NOALLOC_MAX_EDITS
    for n_ins, n_del in ((cap + 1, 0), (0, cap + 1), (cap, 1), (2**64 - 1, 1), (1, 2**64 - 1)):
        assert lib.cgb_merge_keys_noalloc(None, 0, p, n_ins, p, n_del, 10, p, p, None) == 4, (n_ins, n_del)
    assert lib.cgb_merge_keys_noalloc(None, 0, p, 1, p, 0, 10, None, p, None) == 1
    assert lib.cgb_merge_keys_noalloc(None, 5, p, 1, p, 0, 10, p, p, None) == 1
    # old keys + edits beyond the tile counts the scratch holds (CGB_NOALLOC_MAX_KEYS)
    keys = engine.NOALLOC_MAX_KEYS
    for n_old, n_ins in ((keys, 1), (keys - 5, 6), (2**64 - 1, 1)):
        assert lib.cgb_merge_keys_noalloc(p, n_old, p, n_ins, None, 0, 10, p, p, None) == 4, (n_old, n_ins)
