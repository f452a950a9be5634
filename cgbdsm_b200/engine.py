"""ctypes binding of the engine's C ABI (include/cgbdsm.h).

The engine itself is native (CUDA + C++ in libcgbdsm.so); this module only
marshals arrays.  There is no Python or CPU fallback: if the shared library
is missing or no CUDA device is present, construction raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcgbdsm.so")

_u32, _u64, _vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_OOM", 4: "ERR_LIMIT", 5: "ERR_STATE",
          6: "ERR_TIMEOUT", 7: "ERR_IO"}

# Every entry point declared in include/cgbdsm.h (checked by tests/test_abi.py).
EXPORTS = [
    "cgb_default_config", "cgb_create", "cgb_destroy", "cgb_last_error", "cgb_load_query",
    "cgb_load_query_file", "cgb_query_dir", "cgb_build_index", "cgb_apply_batch",
    "cgb_apply_batch_device", "cgb_last_edge_counts", "cgb_read_index", "cgb_last_timings",
    "cgb_kernel_launches", "cgb_last_stats", "cgb_stream", "cgb_plan_anchor", "cgb_plan_info", "cgb_check_symmetry",
    "cgb_producer_open", "cgb_producer_close", "cgb_producer_last_error",
    "cgb_producer_num_batches", "cgb_producer_initial", "cgb_producer_next", "cgb_producer_vertex_map",
    "cgb_merge_keys_noalloc", "cgb_valid_bits", "cgb_starting_edge",
    "cgb_gpma_create", "cgb_gpma_destroy", "cgb_gpma_last_error", "cgb_gpma_bulk_load", "cgb_gpma_batch_update",
    "cgb_gpma_extract", "cgb_gpma_stats",
    "cgb_mq_default_config", "cgb_mq_create", "cgb_mq_destroy", "cgb_mq_last_error", "cgb_mq_load_graph",
    "cgb_mq_register_query", "cgb_mq_unregister_query", "cgb_mq_apply_batch", "cgb_mq_apply_batch_device",
    "cgb_mq_last_timings", "cgb_mq_last_stats", "cgb_mq_query_info", "cgb_mq_schedule", "cgb_mq_kernel_launches",
    "cgb_mq_stream",
    "cgb_server_default_config", "cgb_server_create", "cgb_server_destroy", "cgb_server_last_error",
    "cgb_server_submit_batch", "cgb_server_submit_register", "cgb_server_submit_unregister", "cgb_server_wait",
    "cgb_server_stats",
]

# Edits one cgb_merge_keys_noalloc call accepts (CGB_NOALLOC_MAX_EDITS), and
# old keys + edits (CGB_NOALLOC_MAX_KEYS).
NOALLOC_MAX_EDITS = 1 << 18
NOALLOC_MAX_KEYS = 1 << 27


class CgbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("pool_words", _u64), ("dfs_blocks_per_sm", _u32),
                ("flags", _u32), ("dfs_budget_ms", _u32), ("shard_index", _u32), ("num_shards", _u32)]


FLAG_NO_MERGE_BACK_DEFER = 0x1
FLAG_ENUMERATE_TAIL = 0x2
FLAG_FORCE_SPLIT = 0x4
FLAG_NO_STEAL = 0x8
FLAG_NO_TAIL_CACHE = 0x10
FLAG_PLAIN_CORE_ORDER = 0x20
FLAG_VALID_BITS = 0x40
FLAG_MASK_PRUNE = 0x80
FLAG_NO_SEED_GROUPS = 0x100
FLAG_NO_RUN_BITS = 0x200
FLAG_FOOTPRINT = 0x400
FLAG_WARP_TAIL = 0x800
FLAG_NO_LEVEL_SUM = 0x1000


class MqConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("flags", _u32), ("dfs_budget_ms", _u32), ("dfs_blocks_per_sm", _u32),
                ("pool_words", _u64)]


MQ_FLAG_NO_AUTOTUNE = 0x1
MQ_FLAG_NO_GRAPH = 0x2
MQ_FLAG_NO_RUN_BITS = 0x4
MQ_MAX_QUERIES = 256


class ServerConfig(ctypes.Structure):
    _fields_ = [("mq", MqConfig), ("hbm_budget_bytes", _u64), ("staging_bytes", _u64), ("max_pending", _u32)]


class ServerResult(ctypes.Structure):
    _fields_ = [("ticket", _u64), ("kind", _u32), ("status", ctypes.c_int32), ("query_id", _u32),
                ("live_queries", _u32), ("t_submit_ms", ctypes.c_double), ("t_staged_ms", ctypes.c_double),
                ("t_start_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double), ("device_ms", ctypes.c_float)]


SERVER_BATCH, SERVER_REGISTER, SERVER_UNREGISTER = 0, 1, 2


class BatchKeys(ctypes.Structure):
    _fields_ = [("ins", ctypes.POINTER(_u64)), ("n_ins", _u64), ("dele", ctypes.POINTER(_u64)), ("n_del", _u64),
                ("delta", ctypes.POINTER(_u64)), ("n_delta", _u64), ("edge_ok", ctypes.POINTER(ctypes.c_uint8)),
                ("qe", _u32), ("dv_count", _u32), ("batch", _u32), ("num_edges", _u32),
                ("ms_update_index", ctypes.c_double), ("ms_construct_update", ctypes.c_double),
                ("ms_prepare", ctypes.c_double)]

_lib_handle = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libcgbdsm.so; raises if it has not been built."""
    global _lib_handle
    if _lib_handle is not None:
        return _lib_handle
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built; run `python -m cgbdsm_b200.build`")
    lib = ctypes.CDLL(path)
    lib.cgb_default_config.argtypes = [ctypes.POINTER(Config)]
    lib.cgb_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(_vp)]
    lib.cgb_destroy.argtypes = [_vp]
    lib.cgb_last_error.argtypes = [_vp]
    lib.cgb_last_error.restype = ctypes.c_char_p
    lib.cgb_load_query.argtypes = [_vp, _u32, _vp, _u32, _vp]
    lib.cgb_load_query_file.argtypes = [_vp, ctypes.c_char_p]
    lib.cgb_query_dir.argtypes = [_vp, _u32, _u32]
    lib.cgb_query_dir.restype = _u32
    lib.cgb_build_index.argtypes = [_vp, _vp, _u64, _u32]
    lib.cgb_apply_batch.argtypes = [_vp, _u32, _vp, _u64, _vp, _u64, _vp, _u64, _vp, ctypes.POINTER(_u64)]
    lib.cgb_apply_batch_device.argtypes = [_vp, _u32, _vp, _u64, _vp, _u64, _vp, _u64, _vp, _vp,
                                           ctypes.POINTER(_u64)]
    lib.cgb_last_edge_counts.argtypes = [_vp, _vp, _u32]
    lib.cgb_read_index.argtypes = [_vp, _vp, _u64, ctypes.POINTER(_u64)]
    lib.cgb_last_timings.argtypes = [_vp, _vp]
    lib.cgb_kernel_launches.argtypes = [_vp]
    lib.cgb_kernel_launches.restype = _u64
    lib.cgb_last_stats.argtypes = [_vp, _vp]
    lib.cgb_stream.argtypes = [_vp]
    lib.cgb_stream.restype = _vp
    lib.cgb_plan_anchor.argtypes = [_vp, _u32, ctypes.POINTER(_u32)]
    lib.cgb_plan_info.argtypes = [_vp, _u32, _vp]
    lib.cgb_check_symmetry.argtypes = [_vp, ctypes.POINTER(_u64)]
    lib.cgb_producer_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _u32, _u32,
                                      ctypes.POINTER(_vp)]
    lib.cgb_producer_close.argtypes = [_vp]
    lib.cgb_producer_last_error.argtypes = [_vp]
    lib.cgb_producer_last_error.restype = ctypes.c_char_p
    lib.cgb_producer_num_batches.argtypes = [_vp]
    lib.cgb_producer_num_batches.restype = _u32
    lib.cgb_producer_initial.argtypes = [_vp, ctypes.POINTER(ctypes.POINTER(_u64)), ctypes.POINTER(_u64),
                                         ctypes.POINTER(_u32)]
    lib.cgb_producer_next.argtypes = [_vp, ctypes.POINTER(BatchKeys)]
    lib.cgb_producer_vertex_map.argtypes = [_vp, ctypes.POINTER(ctypes.POINTER(_u32)), ctypes.POINTER(_u32)]
    lib.cgb_merge_keys_noalloc.argtypes = [_vp, _u64, _vp, _u64, _vp, _u64, _u32, _vp, _vp, _vp]
    lib.cgb_valid_bits.argtypes = [_vp, _vp, _u64, ctypes.POINTER(_u64), ctypes.POINTER(ctypes.c_float)]
    lib.cgb_starting_edge.argtypes = [_vp, _vp]
    lib.cgb_gpma_create.argtypes = [ctypes.c_int, _u32, ctypes.POINTER(_vp)]
    lib.cgb_gpma_destroy.argtypes = [_vp]
    lib.cgb_gpma_last_error.argtypes = [_vp]
    lib.cgb_gpma_last_error.restype = ctypes.c_char_p
    lib.cgb_gpma_bulk_load.argtypes = [_vp, _vp, _u64]
    lib.cgb_gpma_batch_update.argtypes = [_vp, _vp, _u64, _vp, _u64]
    lib.cgb_gpma_extract.argtypes = [_vp, _u32, _vp, _u64, ctypes.POINTER(_u64)]
    lib.cgb_gpma_stats.argtypes = [_vp, _vp]
    lib.cgb_mq_default_config.argtypes = [ctypes.POINTER(MqConfig)]
    lib.cgb_mq_create.argtypes = [ctypes.POINTER(MqConfig), ctypes.POINTER(_vp)]
    lib.cgb_mq_destroy.argtypes = [_vp]
    lib.cgb_mq_last_error.argtypes = [_vp]
    lib.cgb_mq_last_error.restype = ctypes.c_char_p
    lib.cgb_mq_load_graph.argtypes = [_vp, _u32, _vp, _u64, _vp]
    lib.cgb_mq_register_query.argtypes = [_vp, _u32, _vp, _u32, _vp, ctypes.POINTER(_u32)]
    lib.cgb_mq_unregister_query.argtypes = [_vp, _u32]
    lib.cgb_mq_apply_batch.argtypes = [_vp, _vp, _u64, _vp, _u64, _vp, _vp, _u32]
    lib.cgb_mq_apply_batch_device.argtypes = [_vp, _vp, _u64, _vp, _u64, _vp, _vp, _vp, _u32]
    lib.cgb_mq_last_timings.argtypes = [_vp, _vp]
    lib.cgb_mq_last_stats.argtypes = [_vp, _vp]
    lib.cgb_mq_query_info.argtypes = [_vp, _u32, ctypes.POINTER(_u32), ctypes.POINTER(ctypes.c_float)]
    lib.cgb_mq_schedule.argtypes = [_vp, ctypes.POINTER(_u32), ctypes.POINTER(_u32)]
    lib.cgb_mq_kernel_launches.argtypes = [_vp]
    lib.cgb_mq_kernel_launches.restype = _u64
    lib.cgb_mq_stream.argtypes = [_vp]
    lib.cgb_mq_stream.restype = _vp
    lib.cgb_server_default_config.argtypes = [ctypes.POINTER(ServerConfig)]
    lib.cgb_server_create.argtypes = [ctypes.POINTER(ServerConfig), _u32, _vp, _u64, _vp, ctypes.POINTER(_vp)]
    lib.cgb_server_destroy.argtypes = [_vp]
    lib.cgb_server_last_error.argtypes = [_vp]
    lib.cgb_server_last_error.restype = ctypes.c_char_p
    lib.cgb_server_submit_batch.argtypes = [_vp, _vp, _u64, _vp, _u64, ctypes.POINTER(_u64)]
    lib.cgb_server_submit_register.argtypes = [_vp, _u32, _vp, _u32, _vp, ctypes.POINTER(_u64)]
    lib.cgb_server_submit_unregister.argtypes = [_vp, _u32, ctypes.POINTER(_u64)]
    lib.cgb_server_wait.argtypes = [_vp, _u64, _u32, ctypes.POINTER(ServerResult), _vp, _vp, _u32]
    lib.cgb_server_stats.argtypes = [_vp, _vp]
    for name in EXPORTS:
        getattr(lib, name)
    _lib_handle = lib
    return lib


def _arr(a: Optional[np.ndarray]) -> tuple[int, int]:
    if a is None or len(a) == 0:
        return 0, 0
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data, len(a)


class Engine:
    """One engine instance on one CUDA device (C ABI handle)."""

    def __init__(self, device: int = 0, pool_words: int = 0, dfs_blocks_per_sm: int = 0, flags: int = 0,
                 dfs_budget_ms: int = 0, shard_index: int = 0, num_shards: int = 1):
        self.lib = load_library()
        cfg = Config(device, pool_words, dfs_blocks_per_sm, flags, dfs_budget_ms, shard_index, num_shards)
        h = _vp()
        st = self.lib.cgb_create(ctypes.byref(cfg), ctypes.byref(h))
        self.h = h.value
        if st != 0:
            msg = self.lib.cgb_last_error(self.h).decode() if self.h else ""
            self.close()
            raise CgbError(st, msg)
        self.qe = 0

    def _check(self, st: int) -> None:
        if st != 0:
            raise CgbError(st, self.lib.cgb_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cgb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_query(self, qv: int, edges: Sequence[tuple[int, int]], labels: Optional[Sequence[int]] = None) -> None:
        e = np.asarray(edges, dtype=np.uint32).reshape(-1)
        lab = None if labels is None else np.asarray(labels, dtype=np.uint32)
        self._check(self.lib.cgb_load_query(self.h, qv, lab.ctypes.data if lab is not None else None,
                                            len(e) // 2, e.ctypes.data))
        self.qe = len(e) // 2

    def load_query_file(self, path: str) -> None:
        self._check(self.lib.cgb_load_query_file(self.h, path.encode()))
        from .workloads import read_query
        _, edges = read_query(path)
        self.qe = len(edges)

    def query_dir(self, a: int, b: int) -> int:
        return self.lib.cgb_query_dir(self.h, a, b)

    def build_index(self, keys: np.ndarray, dv_count: int) -> None:
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        p, n = _arr(keys)
        self._check(self.lib.cgb_build_index(self.h, p, n, dv_count))

    def apply_batch(self, dv_count: int, ins: np.ndarray, dele: np.ndarray, delta: np.ndarray,
                    edge_ok: Optional[np.ndarray] = None) -> int:
        ins = np.ascontiguousarray(ins, dtype=np.uint64)
        dele = np.ascontiguousarray(dele, dtype=np.uint64)
        delta = np.ascontiguousarray(delta, dtype=np.uint64)
        pi, ni = _arr(ins)
        pd, nd = _arr(dele)
        pD, nD = _arr(delta)
        ok = None
        if edge_ok is not None:
            ok = np.ascontiguousarray(edge_ok, dtype=np.uint8)
        out = _u64(0)
        self._check(self.lib.cgb_apply_batch(self.h, dv_count, pi, ni, pd, nd, pD, nD,
                                             ok.ctypes.data if ok is not None else None,
                                             ctypes.byref(out)))
        return out.value

    def apply_batch_device(self, dv_count: int, ins_ptr: int, n_ins: int, del_ptr: int, n_del: int,
                           delta_ptr: int, n_delta: int, stream: int = 0) -> int:
        out = _u64(0)
        self._check(self.lib.cgb_apply_batch_device(self.h, dv_count, ins_ptr, n_ins, del_ptr, n_del,
                                                    delta_ptr, n_delta, None, stream or None,
                                                    ctypes.byref(out)))
        return out.value

    def edge_counts(self) -> np.ndarray:
        out = np.zeros(max(self.qe, 1), dtype=np.uint64)
        self._check(self.lib.cgb_last_edge_counts(self.h, out.ctypes.data, self.qe))
        return out[: self.qe]

    def read_index(self) -> np.ndarray:
        n = _u64(0)
        self._check(self.lib.cgb_read_index(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=np.uint64)
        self._check(self.lib.cgb_read_index(self.h, out.ctypes.data, n.value, ctypes.byref(n)))
        return out[: n.value]

    def timings(self) -> np.ndarray:
        t = np.zeros(4, dtype=np.float32)
        self._check(self.lib.cgb_last_timings(self.h, t.ctypes.data))
        return t

    def stats(self) -> dict:
        out = np.zeros(8, dtype=np.uint64)
        self._check(self.lib.cgb_last_stats(self.h, out.ctypes.data))
        return {"seeds": int(out[0]), "chunks": int(out[1]), "tested": int(out[2]), "tails": int(out[3]),
                "match_bytes": int(out[4]), "update_bytes": int(out[5]), "touched_runs": int(out[6]),
                "stolen_tasks": int(out[7])}

    def valid_bits(self) -> tuple[np.ndarray, float]:
        """Valid bits of the last matched batch, words [ei][u][(dv+31)//32], and the pass's device ms."""
        n = _u64(0)
        ms = ctypes.c_float(0)
        self._check(self.lib.cgb_valid_bits(self.h, None, 0, ctypes.byref(n), ctypes.byref(ms)))
        out = np.zeros(max(n.value, 1), dtype=np.uint32)
        self._check(self.lib.cgb_valid_bits(self.h, out.ctypes.data, n.value, ctypes.byref(n), None))
        return out[: n.value], float(ms.value)

    def starting_edge(self) -> tuple[int, int]:
        out = np.zeros(2, dtype=np.uint32)
        self._check(self.lib.cgb_starting_edge(self.h, out.ctypes.data))
        return int(out[0]), int(out[1])

    def stream(self) -> int:
        return int(self.lib.cgb_stream(self.h) or 0)

    def plan_anchor(self, ei: int) -> int:
        """Query vertex at the first position of query edge ei's plan (keys the seed shard)."""
        v = _u32(0)
        self._check(self.lib.cgb_plan_anchor(self.h, ei, ctypes.byref(v)))
        return v.value

    def plan_info(self, ei: int) -> dict:
        """How query edge ei's plan counts: core positions, first level-sum
        position (0 = none), dense sums, per-lane tail mode, memoized subtree
        (first position, 0 = none; key position)."""
        out = np.zeros(4, dtype=np.uint32)
        self._check(self.lib.cgb_plan_info(self.h, ei, out.ctypes.data))
        return {"n_core": int(out[0]), "sum_from": int(out[1]), "dense": bool(out[2]), "tail_lane": int(out[3] & 0xff),
                "memo_from": int((out[3] >> 8) & 0xff), "memo_pos": int((out[3] >> 16) & 0xff)}

    def check_symmetry(self) -> int:
        """Index entries whose mirror entry is missing (0 for a symmetric index)."""
        n = _u64(0)
        self._check(self.lib.cgb_check_symmetry(self.h, ctypes.byref(n)))
        return n.value

    def kernel_launches(self) -> int:
        return int(self.lib.cgb_kernel_launches(self.h))


def _copy(p, n, dtype=np.uint64) -> np.ndarray:
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(p, (n,)).copy()


class Producer:
    """Stage-1 producer (CaLiG index + host staging) through the C ABI; CPU only."""

    def __init__(self, query: str, data: str, update: str, batch_size_ints: int, threads: int = 0):
        self.lib = load_library()
        h = _vp()
        st = self.lib.cgb_producer_open(query.encode(), data.encode(), update.encode(), batch_size_ints,
                                        threads, ctypes.byref(h))
        self.h = h.value
        if st != 0:
            msg = self.lib.cgb_producer_last_error(self.h).decode() if self.h else ""
            self.close()
            raise CgbError(st, msg)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cgb_producer_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_batches(self) -> int:
        return self.lib.cgb_producer_num_batches(self.h)

    def initial(self) -> tuple[np.ndarray, int]:
        p = ctypes.POINTER(_u64)()
        n = _u64(0)
        dv = _u32(0)
        st = self.lib.cgb_producer_initial(self.h, ctypes.byref(p), ctypes.byref(n), ctypes.byref(dv))
        if st != 0:
            raise CgbError(st, self.lib.cgb_producer_last_error(self.h).decode())
        return _copy(p, n.value), dv.value

    def next(self) -> dict:
        bk = BatchKeys()
        st = self.lib.cgb_producer_next(self.h, ctypes.byref(bk))
        if st != 0:
            raise CgbError(st, self.lib.cgb_producer_last_error(self.h).decode())
        return {"ins": _copy(bk.ins, bk.n_ins), "del": _copy(bk.dele, bk.n_del),
                "delta": _copy(bk.delta, bk.n_delta), "edge_ok": _copy(bk.edge_ok, bk.qe, np.uint8),
                "dv": bk.dv_count, "batch": bk.batch, "num_edges": bk.num_edges,
                "ms": {"update_index": bk.ms_update_index, "construct_update": bk.ms_construct_update,
                       "prepare": bk.ms_prepare}}

    def new2old(self) -> np.ndarray:
        p = ctypes.POINTER(_u32)()
        n = _u32(0)
        self.lib.cgb_producer_vertex_map(self.h, ctypes.byref(p), ctypes.byref(n))
        return _copy(p, n.value, np.uint32)


class Gpma:
    """Packed-memory-array index layout (cgb_gpma_*); key arrays live on the
    device (torch tensors of int64 holding the u64 keys)."""

    def __init__(self, num_dirs: int, device: int = 0):
        self.lib = load_library()
        h = _vp()
        st = self.lib.cgb_gpma_create(device, num_dirs, ctypes.byref(h))
        self.h = h.value
        self.device = device
        if st != 0:
            msg = self.lib.cgb_gpma_last_error(self.h).decode() if self.h else ""
            self.close()
            raise CgbError(st, msg)

    def _check(self, st: int) -> None:
        if st != 0:
            raise CgbError(st, self.lib.cgb_gpma_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cgb_gpma_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dev(self, keys: np.ndarray):
        import torch

        a = np.ascontiguousarray(keys, dtype=np.uint64).view(np.int64)
        return torch.from_numpy(a).to(f"cuda:{self.device}")

    def bulk_load(self, keys: np.ndarray) -> None:
        t = self._dev(keys)
        self._check(self.lib.cgb_gpma_bulk_load(self.h, t.data_ptr() if len(t) else None, len(t)))

    def batch_update(self, ins: np.ndarray, dele: np.ndarray) -> None:
        ti, td = self._dev(ins), self._dev(dele)
        self._check(self.lib.cgb_gpma_batch_update(self.h, ti.data_ptr() if len(ti) else None, len(ti),
                                                   td.data_ptr() if len(td) else None, len(td)))

    def extract(self, d: int) -> np.ndarray:
        """Keys of direction d, ascending, as (u << 32 | v)."""
        import torch

        n = _u64(0)
        self._check(self.lib.cgb_gpma_extract(self.h, d, None, 0, ctypes.byref(n)))
        out = torch.empty(max(n.value, 1), dtype=torch.int64, device=f"cuda:{self.device}")
        self._check(self.lib.cgb_gpma_extract(self.h, d, out.data_ptr(), n.value, ctypes.byref(n)))
        return out[: n.value].cpu().numpy().view(np.uint64)

    def stats(self) -> dict:
        out = np.zeros(6, dtype=np.uint64)
        self._check(self.lib.cgb_gpma_stats(self.h, out.ctypes.data))
        return {"slots": int(out[0]), "windows": int(out[1]), "rewritten": int(out[2]), "rebuilt": int(out[3]),
                "device_us": int(out[4]), "keys": int(out[5])}



def _pairs(edges) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1, 2))
    return a


class MultiQuery:
    """Multi-query engine (cgb_mq_*): one device-resident data-graph index
    shared by registered queries, all matched per batch in one launch."""

    def __init__(self, device: int = 0, flags: int = 0, dfs_budget_ms: int = 0, dfs_blocks_per_sm: int = 0,
                 pool_words: int = 0):
        self.lib = load_library()
        cfg = MqConfig(device, flags, dfs_budget_ms, dfs_blocks_per_sm, pool_words)
        h = _vp()
        st = self.lib.cgb_mq_create(ctypes.byref(cfg), ctypes.byref(h))
        self.h = h.value
        if st != 0:
            msg = self.lib.cgb_mq_last_error(self.h).decode() if self.h else ""
            self.close()
            raise CgbError(st, msg)
        self.ids: set[int] = set()

    def _check(self, st: int) -> None:
        if st != 0:
            raise CgbError(st, self.lib.cgb_mq_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cgb_mq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_graph(self, labels, edges) -> None:
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        e = _pairs(edges)
        self._check(self.lib.cgb_mq_load_graph(self.h, len(lab), lab.ctypes.data, len(e),
                                               e.ctypes.data if len(e) else None))

    def register(self, qv: int, edges, labels) -> int:
        e = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1))
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        qid = _u32(0)
        self._check(self.lib.cgb_mq_register_query(self.h, qv, lab.ctypes.data, len(e) // 2, e.ctypes.data,
                                                   ctypes.byref(qid)))
        self.ids.add(qid.value)
        return qid.value

    def unregister(self, qid: int) -> None:
        self._check(self.lib.cgb_mq_unregister_query(self.h, qid))
        self.ids.discard(qid)

    def apply_batch(self, ins=None, dele=None) -> tuple[np.ndarray, np.ndarray]:
        """(positive, negative) counts per query id (arrays of MQ_MAX_QUERIES u64)."""
        ins = _pairs(ins if ins is not None else np.zeros((0, 2)))
        dele = _pairs(dele if dele is not None else np.zeros((0, 2)))
        pos = np.zeros(MQ_MAX_QUERIES, dtype=np.uint64)
        neg = np.zeros(MQ_MAX_QUERIES, dtype=np.uint64)
        self._check(self.lib.cgb_mq_apply_batch(self.h, ins.ctypes.data if len(ins) else None, len(ins),
                                                dele.ctypes.data if len(dele) else None, len(dele),
                                                pos.ctypes.data, neg.ctypes.data, MQ_MAX_QUERIES))
        return pos, neg

    def apply_batch_device(self, ins_ptr: int, n_ins: int, del_ptr: int = 0, n_del: int = 0,
                           stream: int = 0) -> tuple[np.ndarray, np.ndarray]:
        pos = np.zeros(MQ_MAX_QUERIES, dtype=np.uint64)
        neg = np.zeros(MQ_MAX_QUERIES, dtype=np.uint64)
        self._check(self.lib.cgb_mq_apply_batch_device(self.h, ins_ptr or None, n_ins, del_ptr or None, n_del,
                                                       stream or None, pos.ctypes.data, neg.ctypes.data,
                                                       MQ_MAX_QUERIES))
        return pos, neg

    def timings(self) -> np.ndarray:
        t = np.zeros(4, dtype=np.float32)
        self._check(self.lib.cgb_mq_last_timings(self.h, t.ctypes.data))
        return t

    def stats(self) -> dict:
        out = np.zeros(8, dtype=np.uint64)
        self._check(self.lib.cgb_mq_last_stats(self.h, out.ctypes.data))
        return {"seeds": int(out[0]), "chunks": int(out[1]), "tested": int(out[2]), "tails": int(out[3]),
                "match_bytes": int(out[4]), "update_bytes": int(out[5]), "touched_runs": int(out[6]),
                "stolen_tasks": int(out[7])}

    def query_info(self, qid: int) -> tuple[int, float]:
        v, ms = _u32(0), ctypes.c_float(0)
        self._check(self.lib.cgb_mq_query_info(self.h, qid, ctypes.byref(v), ctypes.byref(ms)))
        return v.value, float(ms.value)

    def schedule(self) -> tuple[int, int]:
        b, st = _u32(0), _u32(0)
        self._check(self.lib.cgb_mq_schedule(self.h, ctypes.byref(b), ctypes.byref(st)))
        return b.value, st.value

    def kernel_launches(self) -> int:
        return int(self.lib.cgb_mq_kernel_launches(self.h))

    def stream(self) -> int:
        return int(self.lib.cgb_mq_stream(self.h) or 0)


class Server:
    """Serving loop (cgb_server_*): graph, index and queries resident on the
    device; update batches and query registrations submitted from any thread,
    applied in submission order, results collected per ticket."""

    def __init__(self, labels, edges, device: int = 0, hbm_budget_bytes: int = 0, staging_bytes: int = 0,
                 max_pending: int = 0, mq_flags: int = 0, dfs_budget_ms: int = 0):
        self.lib = load_library()
        cfg = ServerConfig()
        self.lib.cgb_server_default_config(ctypes.byref(cfg))
        cfg.mq.device = device
        cfg.mq.flags = mq_flags
        cfg.mq.dfs_budget_ms = dfs_budget_ms
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.staging_bytes = staging_bytes
        cfg.max_pending = max_pending
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        e = _pairs(edges)
        h = _vp()
        st = self.lib.cgb_server_create(ctypes.byref(cfg), len(lab), lab.ctypes.data, len(e),
                                        e.ctypes.data if len(e) else None, ctypes.byref(h))
        self.h = h.value
        if st != 0:
            msg = self.lib.cgb_server_last_error(self.h).decode() if self.h else ""
            self.close()
            raise CgbError(st, msg)

    def _check(self, st: int) -> None:
        if st != 0:
            raise CgbError(st, self.lib.cgb_server_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cgb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit_batch(self, ins=None, dele=None) -> int:
        ins = _pairs(ins if ins is not None else np.zeros((0, 2)))
        dele = _pairs(dele if dele is not None else np.zeros((0, 2)))
        t = _u64(0)
        self._check(self.lib.cgb_server_submit_batch(self.h, ins.ctypes.data if len(ins) else None, len(ins),
                                                     dele.ctypes.data if len(dele) else None, len(dele),
                                                     ctypes.byref(t)))
        return t.value

    def submit_register(self, qv: int, edges, labels) -> int:
        e = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1))
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        t = _u64(0)
        self._check(self.lib.cgb_server_submit_register(self.h, qv, lab.ctypes.data, len(e) // 2, e.ctypes.data,
                                                        ctypes.byref(t)))
        return t.value

    def submit_unregister(self, qid: int) -> int:
        t = _u64(0)
        self._check(self.lib.cgb_server_submit_unregister(self.h, qid, ctypes.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 600000) -> dict:
        """Result of a request: status, timestamps, query id (registrations),
        counts per query id (batches)."""
        res = ServerResult()
        pos = np.zeros(MQ_MAX_QUERIES, dtype=np.uint64)
        neg = np.zeros(MQ_MAX_QUERIES, dtype=np.uint64)
        self._check(self.lib.cgb_server_wait(self.h, ticket, timeout_ms, ctypes.byref(res), pos.ctypes.data,
                                             neg.ctypes.data, MQ_MAX_QUERIES))
        err = self.lib.cgb_server_last_error(self.h).decode() if res.status != 0 else ""
        return {"ticket": res.ticket, "kind": res.kind, "status": res.status, "error": err, "query_id": res.query_id,
                "live_queries": res.live_queries, "t_submit_ms": res.t_submit_ms, "t_staged_ms": res.t_staged_ms,
                "t_start_ms": res.t_start_ms, "t_done_ms": res.t_done_ms, "device_ms": res.device_ms,
                "pos": pos, "neg": neg}

    def stats(self) -> dict:
        out = np.zeros(8, dtype=np.uint64)
        self._check(self.lib.cgb_server_stats(self.h, out.ctypes.data))
        keys = ["batches_done", "edges_done", "rejected", "live_queries", "queued", "staging_bytes",
                "hbm_budget_bytes", "busy_us"]
        return {k: int(v) for k, v in zip(keys, out)}
