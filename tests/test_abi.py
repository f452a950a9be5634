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
