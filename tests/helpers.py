"""Shared fixtures of the test suite: small seeded workloads and comparison helpers."""
import numpy as np

from csm import Batch, DataGraph, QueryGraph, gen


def small_workload(name="c1", scale=1.0, seed=None, nqueries=None, n_del=None, batch=None):
    cfg = gen.scaled(name, scale) if scale != 1.0 else dict(gen.CONFIGS[name])
    if n_del is not None:
        cfg["n_del"] = n_del
    if batch is not None:
        cfg["batch"] = batch
    return gen.make_workload(name, cfg, seed=seed, nqueries=nqueries)


def random_graph(n, m, nlab, rng, nel=1):
    s = rng.integers(0, n, size=m * 2)
    d = rng.integers(0, n, size=m * 2)
    ok = s != d
    lo, hi = np.minimum(s[ok], d[ok]), np.maximum(s[ok], d[ok])
    keys = np.unique(lo.astype(np.int64) * n + hi)[:m]
    rng.shuffle(keys)
    src = (keys // n).astype(np.uint32)
    dst = (keys % n).astype(np.uint32)
    el = rng.integers(0, nel, size=len(src)).astype(np.uint32)
    vl = rng.integers(0, nlab, size=n).astype(np.uint32)
    return vl, src, dst, el


def clique(k, label=0):
    s, d = zip(*[(i, j) for i in range(k) for j in range(i + 1, k)])
    return QueryGraph(np.full(k, label, dtype=np.uint32), np.array(s, dtype=np.uint32), np.array(d, dtype=np.uint32),
                      np.zeros(len(s), dtype=np.uint32))


def cycle(k, labels=None):
    labels = np.zeros(k, dtype=np.uint32) if labels is None else np.asarray(labels, dtype=np.uint32)
    return QueryGraph(labels, np.arange(k, dtype=np.uint32), (np.arange(k, dtype=np.uint32) + 1) % k,
                      np.zeros(k, dtype=np.uint32))


def star(k, center=0, leaf=0):
    return QueryGraph(np.array([center] + [leaf] * k, dtype=np.uint32), np.zeros(k, dtype=np.uint32),
                      np.arange(1, k + 1, dtype=np.uint32), np.zeros(k, dtype=np.uint32))


def path(k):
    return QueryGraph(np.zeros(k, dtype=np.uint32), np.arange(k - 1, dtype=np.uint32),
                      np.arange(1, k, dtype=np.uint32), np.zeros(k - 1, dtype=np.uint32))
