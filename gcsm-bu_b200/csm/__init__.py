"""Python host mirror of the csmg / libcsm interface (ctypes over include/csm.h).

The reference (gh8li/GCSM-BU) is driven by its `csmg` process: main.cpp:162-190 parses the
flags, technique_permutation.h:29-225 loads the query, the data graph and the update stream and
runs the per-batch loop.  `Engine` exposes the same steps as methods over libcsm.so, and
`run_csmg_like` replays a whole stream the way the reference's driver does.

The CUDA library is the only compute path: importing this module on a machine without the
built library, or calling it without a B200, raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libcsm.so")
CSMG_PATH = os.path.join(os.path.dirname(_HERE), "bin", "csmg")

CSM_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of memory",
    -4: "timeout",
    -5: "bad state",
    -6: "limit exceeded",
    -7: "overflow",
    -8: "no device",
}

# Every symbol declared in include/csm.h.
EXPORTED = [
    "csm_default_config", "csm_create", "csm_destroy", "csm_load_query", "csm_load_graph",
    "csm_save_snapshot", "csm_load_snapshot",
    "csm_apply_batch", "csm_apply_batch_device", "csm_apply_batch_device_static", "csm_set_time_limit",
    "csm_get_edge_counts", "csm_get_embeddings",
    "csm_free", "csm_describe_plan", "csm_get_stats", "csm_reset_stats", "csm_device_memory",
    "csm_last_error", "csm_version",
]

# Every symbol declared in include/csm_server.h.
SERVER_EXPORTED = [
    "csm_server_default_config", "csm_server_create", "csm_server_add_tenant", "csm_server_submit",
    "csm_server_wait", "csm_server_get_stats", "csm_server_destroy", "csm_server_last_error",
]


class CsmConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("algorithm", ctypes.c_int32),
        ("matching_order", ctypes.c_int32),
        ("search_strategy", ctypes.c_int32),
        ("local_index", ctypes.c_int32),
        ("cartesian_product", ctypes.c_int32),
        ("heavy_vertex_avoidance", ctypes.c_int32),
        ("relation_switch", ctypes.c_int32),
        ("pool_entries", ctypes.c_uint64),
        ("max_batch", ctypes.c_uint64),
        ("frontier_bytes", ctypes.c_uint64),
        ("materialize_rows", ctypes.c_uint64),
        ("blocks_per_sm", ctypes.c_int32),
        ("warps_per_block", ctypes.c_int32),
        ("steal_chunk", ctypes.c_int32),
        ("occupancy", ctypes.c_int32),
        ("autotune_batches", ctypes.c_int32),
        ("cuda_graphs", ctypes.c_int32),
        ("replan_drift_pct", ctypes.c_int32),
        ("semi_bfs_items_per_warp", ctypes.c_int32),
        ("queue_slots", ctypes.c_int32),
        ("inject_alloc_failure", ctypes.c_int32),
        ("time_limit_us", ctypes.c_uint64),
    ]


class CsmBatchResult(ctypes.Structure):
    _fields_ = [
        ("positive", ctypes.c_uint64),
        ("negative", ctypes.c_uint64),
        ("inserted", ctypes.c_uint64),
        ("deleted", ctypes.c_uint64),
        ("latency_ns", ctypes.c_uint64),
        ("apply_ns", ctypes.c_uint64),
        ("enum_ns", ctypes.c_uint64),
        ("reserved", ctypes.c_uint64),
    ]


class CsmStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "batches", "enum_launches", "kernel_launches", "enum_scan_entries", "enum_probes",
        "enum_tail_lists", "donations", "enum_ns", "apply_ns", "pool_used", "pool_capacity",
        "compactions", "tuned_strategy", "tuned_steal_chunk", "tuned_warps_per_block", "tuned_occupancy",
        "graph_launches", "replans", "donations_refused", "enum_shared_last")]


class CsmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"csm error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


class CsmServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("slots", ctypes.c_int32),
        ("memory_budget", ctypes.c_uint64),
        ("min_frontier_bytes", ctypes.c_uint64),
        ("max_pending", ctypes.c_uint32),
        ("reserved", ctypes.c_int32 * 7),
    ]


class CsmRequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("nresults", ctypes.c_uint32)] + [
        (n, ctypes.c_uint64) for n in ("arrival_ns", "start_ns", "done_ns", "frontier_bytes", "device_ns")] + [
        ("reserved", ctypes.c_uint64 * 2)]


class CsmServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "requests", "units", "units_depth_first", "units_shrunk", "memory_waits", "peak_frontier_bytes",
        "peak_inflight")] + [("reserved", ctypes.c_uint64 * 5)]


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libcsm.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `make -C gcsm-bu_b200`")
    lib = ctypes.CDLL(path)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    u8p = ctypes.POINTER(ctypes.c_uint8)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    vp = ctypes.c_void_p
    lib.csm_version.restype = ctypes.c_char_p
    lib.csm_default_config.argtypes = [ctypes.POINTER(CsmConfig)]
    lib.csm_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(CsmConfig)]
    lib.csm_destroy.argtypes = [vp]
    lib.csm_load_query.argtypes = [vp, ctypes.c_uint32, u32p, ctypes.c_uint32, u32p, u32p, u32p,
                                   ctypes.POINTER(ctypes.c_int32)]
    lib.csm_load_graph.argtypes = [vp, ctypes.c_uint32, u32p, ctypes.c_uint64, u32p, u32p, u32p]
    lib.csm_save_snapshot.argtypes = [vp, ctypes.c_char_p]
    lib.csm_load_snapshot.argtypes = [vp, ctypes.c_char_p]
    lib.csm_apply_batch.argtypes = [vp, ctypes.c_uint64, u32p, u32p, u32p, u8p, ctypes.POINTER(CsmBatchResult)]
    lib.csm_apply_batch_device.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp, vp, ctypes.POINTER(CsmBatchResult)]
    lib.csm_apply_batch_device_static.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp, vp,
                                                  ctypes.POINTER(CsmBatchResult)]
    lib.csm_set_time_limit.argtypes = [vp, ctypes.c_uint64]
    lib.csm_get_edge_counts.argtypes = [vp, ctypes.c_int32, u64p, u64p, ctypes.c_uint32, u32p]
    lib.csm_get_embeddings.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(u32p), u64p]
    lib.csm_free.argtypes = [vp]
    lib.csm_describe_plan.argtypes = [vp, ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t]
    lib.csm_get_stats.argtypes = [vp, ctypes.POINTER(CsmStats)]
    lib.csm_reset_stats.argtypes = [vp]
    lib.csm_device_memory.argtypes = [vp, u64p, u64p]
    lib.csm_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.csm_server_default_config.argtypes = [ctypes.POINTER(CsmServerConfig)]
    lib.csm_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(CsmServerConfig)]
    lib.csm_server_add_tenant.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_int32)]
    lib.csm_server_submit.argtypes = [vp, ctypes.c_int32, ctypes.c_uint64, u32p, u32p, u32p, u8p, u64p]
    lib.csm_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(CsmRequestInfo),
                                    ctypes.POINTER(CsmBatchResult), ctypes.c_uint32]
    lib.csm_server_get_stats.argtypes = [vp, ctypes.POINTER(CsmServerStats)]
    lib.csm_server_destroy.argtypes = [vp]
    lib.csm_server_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    for name in EXPORTED + SERVER_EXPORTED:
        if name != "csm_version":
            getattr(lib, name).restype = ctypes.c_int32
    _lib = lib
    return lib


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _ptr(a: np.ndarray, ctype=ctypes.c_uint32):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def default_config(**overrides) -> CsmConfig:
    lib = load_library()
    cfg = CsmConfig()
    lib.csm_default_config(ctypes.byref(cfg))
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


@dataclass
class QueryGraph:
    """A labelled query: vertices 0..nv-1 with labels, undirected labelled edges."""
    vlabels: np.ndarray
    src: np.ndarray
    dst: np.ndarray
    elabels: np.ndarray

    @property
    def nv(self) -> int:
        return int(len(self.vlabels))


@dataclass
class DataGraph:
    vlabels: np.ndarray
    src: np.ndarray
    dst: np.ndarray
    elabels: np.ndarray


@dataclass
class Batch:
    src: np.ndarray
    dst: np.ndarray
    elabels: np.ndarray
    is_delete: Optional[np.ndarray] = None


class Engine:
    """One libcsm engine on one GPU (csm_create .. csm_destroy)."""

    def __init__(self, config: Optional[CsmConfig] = None, **overrides):
        self.lib = load_library()
        cfg = config if config is not None else default_config()
        for k, v in overrides.items():
            setattr(cfg, k, v)
        self.config = cfg
        self._h = ctypes.c_void_p()
        rc = self.lib.csm_create(ctypes.byref(self._h), ctypes.byref(cfg))
        if rc != CSM_OK:
            raise CsmError(rc, self._err(None))
        self.queries: List[QueryGraph] = []

    def _err(self, h) -> str:
        buf = ctypes.create_string_buffer(1024)
        self.lib.csm_last_error(h, buf, len(buf))
        return buf.value.decode(errors="replace")

    def _check(self, rc: int):
        if rc != CSM_OK:
            raise CsmError(rc, self._err(self._h))

    def close(self):
        if self._h:
            self.lib.csm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_query(self, q: QueryGraph) -> int:
        vl, s, d, l = _u32(q.vlabels), _u32(q.src), _u32(q.dst), _u32(q.elabels)
        qid = ctypes.c_int32(-1)
        self._check(self.lib.csm_load_query(self._h, len(vl), _ptr(vl), len(s), _ptr(s), _ptr(d), _ptr(l),
                                            ctypes.byref(qid)))
        self.queries.append(q)
        return qid.value

    def load_graph(self, g: DataGraph):
        vl, s, d, l = _u32(g.vlabels), _u32(g.src), _u32(g.dst), _u32(g.elabels)
        self._check(self.lib.csm_load_graph(self._h, len(vl), _ptr(vl), len(s), _ptr(s), _ptr(d), _ptr(l)))

    def save_snapshot(self, path: str):
        """csm_save_snapshot: the data graph after the last batch, to a binary file."""
        self._check(self.lib.csm_save_snapshot(self._h, os.fsencode(path)))

    def load_snapshot(self, path: str):
        """csm_load_snapshot: restores a snapshot instead of load_graph (same queries first)."""
        self._check(self.lib.csm_load_snapshot(self._h, os.fsencode(path)))

    def apply(self, b: Batch) -> List[CsmBatchResult]:
        s, d, l = _u32(b.src), _u32(b.dst), _u32(b.elabels)
        out = (CsmBatchResult * max(1, len(self.queries)))()
        dp = None
        if b.is_delete is not None:
            dl = np.ascontiguousarray(np.asarray(b.is_delete, dtype=np.uint8))
            dp = _ptr(dl, ctypes.c_uint8)
        self._check(self.lib.csm_apply_batch(self._h, len(s), _ptr(s), _ptr(d), _ptr(l), dp, out))
        return list(out)[: len(self.queries)]

    def apply_device(self, n: int, src_ptr: int, dst_ptr: int, lab_ptr: int, del_ptr: Optional[int] = None,
                     stream: Optional[int] = None) -> List[CsmBatchResult]:
        out = (CsmBatchResult * max(1, len(self.queries)))()
        self._check(self.lib.csm_apply_batch_device(self._h, n, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                                    ctypes.c_void_p(lab_ptr),
                                                    ctypes.c_void_p(del_ptr) if del_ptr else None,
                                                    ctypes.c_void_p(stream) if stream else None, out))
        return list(out)[: len(self.queries)]

    def apply_device_static(self, n: int, src_ptr: int, dst_ptr: int, lab_ptr: int, del_ptr: Optional[int] = None,
                            stream: Optional[int] = None) -> List[CsmBatchResult]:
        """csm_apply_batch_device_static: the same batch, allocating nothing during the call."""
        out = (CsmBatchResult * max(1, len(self.queries)))()
        self._check(self.lib.csm_apply_batch_device_static(
            self._h, n, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr), ctypes.c_void_p(lab_ptr),
            ctypes.c_void_p(del_ptr) if del_ptr else None, ctypes.c_void_p(stream) if stream else None, out))
        return list(out)[: len(self.queries)]

    def set_time_limit(self, us: int):
        """csm_set_time_limit: enumeration launches of later batches stop after `us` microseconds."""
        self._check(self.lib.csm_set_time_limit(self._h, us))

    def apply_partial(self, b: Batch):
        """Like apply(), but returns (status, results): CSM_ERR_TIMEOUT comes back with the partial
        counts instead of raising."""
        s, d, l = _u32(b.src), _u32(b.dst), _u32(b.elabels)
        out = (CsmBatchResult * max(1, len(self.queries)))()
        dp = None
        if b.is_delete is not None:
            dl = np.ascontiguousarray(np.asarray(b.is_delete, dtype=np.uint8))
            dp = _ptr(dl, ctypes.c_uint8)
        rc = self.lib.csm_apply_batch(self._h, len(s), _ptr(s), _ptr(d), _ptr(l), dp, out)
        if rc not in (CSM_OK, -4):
            self._check(rc)
        return rc, list(out)[: len(self.queries)]

    def edge_counts(self, qid: int):
        n = ctypes.c_uint32()
        pos = (ctypes.c_uint64 * 64)()
        neg = (ctypes.c_uint64 * 64)()
        self._check(self.lib.csm_get_edge_counts(self._h, qid, pos, neg, 64, ctypes.byref(n)))
        return list(pos)[: n.value], list(neg)[: n.value]

    def embeddings(self, qid: int, sign: int = 1) -> np.ndarray:
        rows = ctypes.POINTER(ctypes.c_uint32)()
        nrows = ctypes.c_uint64()
        self._check(self.lib.csm_get_embeddings(self._h, qid, sign, ctypes.byref(rows), ctypes.byref(nrows)))
        nv = self.queries[qid].nv
        try:
            if nrows.value == 0:
                return np.zeros((0, nv), dtype=np.uint32)
            arr = np.ctypeslib.as_array(rows, shape=(nrows.value * nv,)).copy()
        finally:
            self.lib.csm_free(rows)
        return arr.reshape(-1, nv)

    def describe(self, qid: int) -> str:
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self.lib.csm_describe_plan(self._h, qid, buf, len(buf)))
        return buf.value.decode()

    def stats(self) -> CsmStats:
        st = CsmStats()
        self._check(self.lib.csm_get_stats(self._h, ctypes.byref(st)))
        return st

    def reset_stats(self):
        self._check(self.lib.csm_reset_stats(self._h))


class Server:
    """Continuous-batching serving loop (include/csm_server.h): tenant engines on one GPU, work
    units admitted to slots as slots and frontier memory free up."""

    def __init__(self, device: int = 0, slots: int = 4, memory_budget: int = 8 << 30,
                 min_frontier_bytes: int = 16 << 20, max_pending: int = 4096):
        self.lib = load_library()
        cfg = CsmServerConfig()
        self.lib.csm_server_default_config(ctypes.byref(cfg))
        cfg.device, cfg.slots, cfg.memory_budget = device, slots, memory_budget
        cfg.min_frontier_bytes, cfg.max_pending = min_frontier_bytes, max_pending
        self._h = ctypes.c_void_p()
        rc = self.lib.csm_server_create(ctypes.byref(self._h), ctypes.byref(cfg))
        if rc != CSM_OK:
            raise CsmError(rc, self._err(None))
        self.tenants: List[Engine] = []
        self._nres = {}

    def _err(self, h) -> str:
        buf = ctypes.create_string_buffer(1024)
        self.lib.csm_server_last_error(h, buf, len(buf))
        return buf.value.decode(errors="replace")

    def _check(self, rc: int):
        if rc != CSM_OK:
            raise CsmError(rc, self._err(self._h))

    def add_tenant(self, eng: Engine) -> int:
        tid = ctypes.c_int32(-1)
        self._check(self.lib.csm_server_add_tenant(self._h, eng._h, ctypes.byref(tid)))
        self.tenants.append(eng)
        return tid.value

    def submit(self, b: Batch, tenant: int = -1) -> int:
        s, d, l = _u32(b.src), _u32(b.dst), _u32(b.elabels)
        dp = None
        if b.is_delete is not None:
            dl = np.ascontiguousarray(np.asarray(b.is_delete, dtype=np.uint8))
            dp = _ptr(dl, ctypes.c_uint8)
        rid = ctypes.c_uint64()
        self._check(self.lib.csm_server_submit(self._h, tenant, len(s), _ptr(s), _ptr(d), _ptr(l), dp,
                                               ctypes.byref(rid)))
        ts = self.tenants if tenant < 0 else [self.tenants[tenant]]
        self._nres[rid.value] = sum(len(t.queries) for t in ts)
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1):
        """Returns (info, per-query results), or None if the request is still running."""
        n = self._nres.get(rid, 0)
        out = (CsmBatchResult * max(1, n))()
        info = CsmRequestInfo()
        rc = self.lib.csm_server_wait(self._h, rid, timeout_ms, ctypes.byref(info), out, n)
        if rc == -4:
            return None
        self._nres.pop(rid, None)
        self._check(rc)
        return info, list(out)[:n]

    def stats(self) -> CsmServerStats:
        st = CsmServerStats()
        self._check(self.lib.csm_server_get_stats(self._h, ctypes.byref(st)))
        return st

    def close(self):
        if self._h:
            self.lib.csm_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def version() -> str:
    return load_library().csm_version().decode()


def run_csmg_like(query: QueryGraph, data: DataGraph, batches: Sequence[Batch], **config) -> List[List[CsmBatchResult]]:
    """Replays a stream the way technique_permutation.h:29-225 does: load, then one call per batch."""
    with Engine(**config) as eng:
        eng.load_query(query)
        eng.load_graph(data)
        return [eng.apply(b) for b in batches]
