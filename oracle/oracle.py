"""ctypes wrapper of liboracle.so — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, as the
checker of the CUDA engine; the engine never routes through it.  The algorithm is restated in
oracle.c (see its header for the reference files it follows).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.c")):
        build()
    lib = ctypes.CDLL(LIB)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    u8p = ctypes.POINTER(ctypes.c_uint8)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    lib.oracle_create.restype = ctypes.c_void_p
    lib.oracle_create.argtypes = [ctypes.c_uint32, u32p, ctypes.c_uint32, u32p, u32p, u32p, ctypes.c_uint32, u32p,
                                  ctypes.c_uint64, u32p, u32p, u32p]
    lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_apply.restype = ctypes.c_int
    lib.oracle_apply.argtypes = [ctypes.c_void_p, ctypes.c_uint64, u32p, u32p, u32p, u8p, ctypes.c_int, ctypes.c_int,
                                 u64p, u64p]
    lib.oracle_apply_sample.restype = ctypes.c_int
    lib.oracle_apply_sample.argtypes = [ctypes.c_void_p, ctypes.c_uint64, u32p, u32p, u32p, u8p, ctypes.c_int,
                                        ctypes.c_double, u64p, u64p]
    lib.oracle_rows.restype = ctypes.c_uint64
    lib.oracle_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, u32p, ctypes.c_uint64]
    lib.oracle_work.argtypes = [ctypes.c_void_p, u64p, u64p]
    lib.oracle_count_all.restype = ctypes.c_uint64
    lib.oracle_count_all.argtypes = [ctypes.c_void_p]
    _lib = lib
    return lib


def _a(x, dt=np.uint32):
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


def _p(a, ct=ctypes.c_uint32):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class Oracle:
    """Stateful CPU oracle: one query, one data graph, batches applied in order."""

    def __init__(self, query, data, nv: Optional[int] = None):
        lib = load()
        self.lib = lib
        self.qn = int(len(query.vlabels))
        self.qm = int(len(query.src))
        ql, qs, qd, qe = _a(query.vlabels), _a(query.src), _a(query.dst), _a(query.elabels)
        vl = _a(data.vlabels)
        s, d, l = _a(data.src), _a(data.dst), _a(data.elabels)
        self._keep = (ql, qs, qd, qe, vl, s, d, l)
        self.h = lib.oracle_create(self.qn, _p(ql), self.qm, _p(qs), _p(qd), _p(qe), len(vl), _p(vl), len(s), _p(s),
                                   _p(d), _p(l))
        if not self.h:
            raise ValueError("oracle_create rejected the query")

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply(self, batch, threads: int = 0, rows: bool = False):
        """Returns dict(pos, neg, ins, dels, per_qe_pos, per_qe_neg)."""
        threads = threads or (os.cpu_count() or 1)
        s, d, l = _a(batch.src), _a(batch.dst), _a(batch.elabels)
        dp = None
        if batch.is_delete is not None:
            dl = _a(batch.is_delete, np.uint8)
            dp = _p(dl, ctypes.c_uint8)
        out = (ctypes.c_uint64 * 4)()
        per = (ctypes.c_uint64 * (2 * self.qm))()
        rc = self.lib.oracle_apply(self.h, len(s), _p(s), _p(d), _p(l), dp, threads, 1 if rows else 0, out, per)
        if rc != 0:
            raise MemoryError("oracle_apply failed")
        return dict(pos=out[0], neg=out[1], ins=out[2], dels=out[3], per_qe_pos=list(per)[: self.qm],
                    per_qe_neg=list(per)[self.qm:])

    def apply_sample(self, batch, max_seconds: float, threads: int = 0):
        """Applies `batch`, counting for at most `max_seconds`; returns (matches, items_done)."""
        threads = threads or (os.cpu_count() or 1)
        s, d, l = _a(batch.src), _a(batch.dst), _a(batch.elabels)
        dp = None
        if batch.is_delete is not None:
            dl = _a(batch.is_delete, np.uint8)
            dp = _p(dl, ctypes.c_uint8)
        out = (ctypes.c_uint64 * 4)()
        items = ctypes.c_uint64()
        rc = self.lib.oracle_apply_sample(self.h, len(s), _p(s), _p(d), _p(l), dp, threads, max_seconds, out,
                                          ctypes.byref(items))
        if rc != 0:
            raise MemoryError("oracle_apply_sample failed")
        return int(out[0] + out[1]), int(items.value)

    def rows(self, sign: int = 1) -> np.ndarray:
        n = self.lib.oracle_rows(self.h, sign, None, 0)
        buf = np.zeros(max(1, n) * self.qn, dtype=np.uint32)
        self.lib.oracle_rows(self.h, sign, _p(buf), n)
        return buf[: n * self.qn].reshape(-1, self.qn)

    def work(self):
        s, p = ctypes.c_uint64(), ctypes.c_uint64()
        self.lib.oracle_work(self.h, ctypes.byref(s), ctypes.byref(p))
        return s.value, p.value

    def count_all(self) -> int:
        return int(self.lib.oracle_count_all(self.h))
