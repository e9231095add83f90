"""Seeded synthetic workloads standing in for the reference's datasets.

The reference's experiments read data graphs and update files that are not part of its
repository (experiments/0_run/run_csm.py:223-224); only the query sets are.  These generators
produce graphs of the shapes the benchmark configurations name: Chung-Lu power-law graphs,
uniform or Zipf vertex labels, an update stream drawn from a held-out 10% of the generated edges
(plus deletions of initial edges), and queries sampled from the data graph so that they match.
Every generator is deterministic in its seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from . import Batch, DataGraph, QueryGraph


def zipf_probs(k: int, s: float) -> np.ndarray:
    p = np.arange(1, k + 1, dtype=np.float64) ** (-s)
    return p / p.sum()


def _sorted_unique(a: np.ndarray) -> np.ndarray:
    """np.unique of an integer array by sorting (numpy's hash-based unique is much slower on
    tens of millions of 64-bit keys); same result."""
    a = np.sort(a)
    if len(a) == 0:
        return a
    keep = np.empty(len(a), dtype=bool)
    keep[0] = True
    np.not_equal(a[1:], a[:-1], out=keep[1:])
    return a[keep]


def chung_lu(n: int, m: int, gamma: float, rng: np.random.Generator, cap: bool = False) -> Tuple[np.ndarray, np.ndarray]:
    """Exactly m distinct undirected edges, endpoints drawn with probability proportional to
    the expected degrees w_k = c (k+1)^(-1/(gamma-1)), with sum(w)/2 = m."""
    w = (np.arange(n, dtype=np.float64) + 1.0) ** (-1.0 / (gamma - 1.0))
    w *= 2.0 * m / w.sum()
    if cap:
        # Structural cutoff of the Chung-Lu model: w_i w_j / sum(w) is an edge probability, so
        # no weight may exceed sqrt(sum(w)).
        w = np.minimum(w, np.sqrt(w.sum()))
    p = w / w.sum()
    cdf = np.cumsum(p)
    cdf[-1] = 1.0
    keys = np.zeros(0, dtype=np.int64)
    need = m
    while need > 0:
        k = int(need * 1.3) + 1024
        a = np.searchsorted(cdf, rng.random(k), side="right")
        b = np.searchsorted(cdf, rng.random(k), side="right")
        a = np.minimum(a, n - 1)
        b = np.minimum(b, n - 1)
        ok = a != b
        lo = np.minimum(a[ok], b[ok]).astype(np.int64)
        hi = np.maximum(a[ok], b[ok]).astype(np.int64)
        keys = _sorted_unique(np.concatenate([keys, lo * n + hi]))
        need = m - len(keys)
    keys = rng.permutation(keys)[:m]
    # Relabel vertices randomly so that hubs are not clustered at small ids.
    perm = rng.permutation(n).astype(np.int64)
    s = perm[keys // n]
    d = perm[keys % n]
    return s.astype(np.uint32), d.astype(np.uint32)


def draw_labels(n: int, k: int, rng: np.random.Generator, zipf: Optional[float]) -> np.ndarray:
    if zipf is None:
        return rng.integers(0, k, size=n).astype(np.uint32)
    return rng.choice(k, size=n, p=zipf_probs(k, zipf)).astype(np.uint32)


class Adjacency:
    """Sorted CSR of an undirected edge list, for query sampling."""

    def __init__(self, n: int, s: np.ndarray, d: np.ndarray, el: np.ndarray):
        a = np.concatenate([s, d]).astype(np.int64)
        b = np.concatenate([d, s]).astype(np.int64)
        l = np.concatenate([el, el])
        # Rows by source, ascending neighbour within a row (a stable sort of one combined key
        # orders like lexsort((b, a))).
        order = np.argsort(a * n + b, kind="stable")
        self.nbr = b[order]
        self.lab = l[order]
        self.off = np.zeros(n + 1, dtype=np.int64)
        self.off[1:] = np.cumsum(np.bincount(a, minlength=n))

    def nbrs(self, v: int) -> np.ndarray:
        return self.nbr[self.off[v]:self.off[v + 1]]

    def edge_label(self, u: int, v: int) -> Optional[int]:
        lo, hi = self.off[u], self.off[u + 1]
        i = lo + np.searchsorted(self.nbr[lo:hi], v)
        if i < hi and self.nbr[i] == v:
            return int(self.lab[i])
        return None


def _induced(adj: Adjacency, vs: List[int], vlab: np.ndarray) -> QueryGraph:
    src, dst, el = [], [], []
    for i in range(len(vs)):
        for j in range(i + 1, len(vs)):
            l = adj.edge_label(vs[i], vs[j])
            if l is not None:
                src.append(i)
                dst.append(j)
                el.append(l)
    return QueryGraph(np.array([vlab[v] for v in vs], dtype=np.uint32), np.array(src, dtype=np.uint32),
                      np.array(dst, dtype=np.uint32), np.array(el, dtype=np.uint32))


def sample_query(adj: Adjacency, vlab: np.ndarray, k: int, kind: str, rng: np.random.Generator,
                 max_tries: int = 400) -> QueryGraph:
    """Samples a connected k-vertex query from the data graph, so that it has matches.

    kind = "tree": a random walk until k distinct vertices are visited; the query is the walk's
    spanning tree.  kind = "sparse": that spanning tree plus 1..k/2 random edges of the data
    graph among the same vertices (so at least one cycle, average degree below 3; walks whose
    vertices span no extra edge are retried).  kind = "dense": the vertex set grows from a random edge, each step adding the
    neighbour with the most edges into the set (ties broken at random), and the query is the
    induced subgraph; sets with average degree >= 3 are preferred (the densest after
    `max_tries` otherwise)."""
    n = len(adj.off) - 1
    deg = np.diff(adj.off)
    starts = np.nonzero(deg > 0)[0]
    best, best_m = None, -1
    for _ in range(max_tries):
        v0 = int(rng.choice(starts))
        if kind == "tree":
            vs, edges, cur, steps = [v0], [], v0, 0
            while len(vs) < k and steps < 50 * k:
                nb = adj.nbrs(cur)
                nxt = int(nb[rng.integers(len(nb))])
                if nxt not in vs:
                    vs.append(nxt)
                    edges.append((vs.index(cur), len(vs) - 1, adj.edge_label(cur, nxt)))
                cur = nxt
                steps += 1
            if len(vs) < k:
                continue
            return QueryGraph(np.array([vlab[v] for v in vs], dtype=np.uint32),
                              np.array([e[0] for e in edges], dtype=np.uint32),
                              np.array([e[1] for e in edges], dtype=np.uint32),
                              np.array([e[2] for e in edges], dtype=np.uint32))
        if kind == "sparse":
            vs, edges, cur, steps = [v0], [], v0, 0
            while len(vs) < k and steps < 50 * k:
                nb = adj.nbrs(cur)
                nxt = int(nb[rng.integers(len(nb))])
                if nxt not in vs:
                    vs.append(nxt)
                    edges.append((vs.index(cur), len(vs) - 1, adj.edge_label(cur, nxt)))
                cur = nxt
                steps += 1
            if len(vs) < k:
                continue
            tree = {(min(a, b), max(a, b)) for a, b, _ in edges}
            ind = _induced(adj, vs, vlab)
            extra = [(int(a), int(b), int(l)) for a, b, l in zip(ind.src, ind.dst, ind.elabels)
                     if (int(a), int(b)) not in tree]
            if not extra:
                continue
            order = rng.permutation(len(extra))
            room = (3 * k - 1) // 2 - (k - 1)
            take = min(len(extra), room, int(rng.integers(1, max(2, k // 2 + 1))))
            edges = edges + [extra[i] for i in order[:take]]
            return QueryGraph(np.array([vlab[v] for v in vs], dtype=np.uint32),
                              np.array([e[0] for e in edges], dtype=np.uint32),
                              np.array([e[1] for e in edges], dtype=np.uint32),
                              np.array([e[2] for e in edges], dtype=np.uint32))
        # dense: a random walk until k distinct vertices, induced subgraph; half of the tries
        # grow greedily instead (most edges into the set), which finds dense sets when walks fail.
        if rng.random() < 0.5:
            vs, cur, steps = [v0], v0, 0
            while len(vs) < k and steps < 50 * k:
                nb = adj.nbrs(cur)
                cur = int(nb[rng.integers(len(nb))])
                if cur not in vs:
                    vs.append(cur)
                steps += 1
            if len(vs) < k:
                continue
            q = _induced(adj, vs, vlab)
            m = len(q.src)
            if 2 * m >= 3 * k:
                return q
            if m > best_m:
                best, best_m = q, m
            continue
        vs = [v0, int(rng.choice(adj.nbrs(v0)))]
        while len(vs) < k:
            cand = {}
            for v in vs:
                nb = adj.nbrs(v)
                if len(nb) > 64:
                    nb = rng.choice(nb, 64, replace=False)
                for w in nb:
                    w = int(w)
                    if w not in vs:
                        cand[w] = cand.get(w, 0) + 1
            if not cand:
                break
            top = max(cand.values())
            pick = [w for w, c in cand.items() if c == top]
            vs.append(int(pick[rng.integers(len(pick))]))
        if len(vs) < k:
            continue
        q = _induced(adj, vs, vlab)
        m = len(q.src)
        if 2 * m >= 3 * k:
            return q
        if m > best_m:
            best, best_m = q, m
    if best is None:
        raise RuntimeError("could not sample a query")
    return best


def expected_batch_matches(q: QueryGraph, vlab: np.ndarray, deg: np.ndarray, n_edges: int, n_updates: int) -> float:
    """Configuration-model estimate of the incremental matches one batch causes for query q.

    With edge (x, y) present with probability deg(x) deg(y) / (2|E|) — the Chung-Lu model with
    the data graph's own degrees — the expected number of embeddings is
        prod_u sum_{v : label(v) = label(u)} deg(v)^{deg_q(u)}  /  (2|E|)^{|E_q|},
    and a batch of n_updates edge updates touches about |E_q| n_updates / |E| of them.
    Injectivity and the cap of each probability at 1 are ignored, so patterns over hubs are
    overestimated (by orders of magnitude); the value ranks queries by cost, it is no count."""
    qdeg = np.bincount(np.concatenate([q.src, q.dst]).astype(np.int64), minlength=q.nv)
    log_total = 0.0
    for u in range(q.nv):
        d = deg[vlab == q.vlabels[u]].astype(np.float64)
        d = d[d > 0]
        if len(d) == 0:
            return 0.0
        ld = np.log(d)
        top = ld.max()
        log_total += qdeg[u] * top + np.log(np.sum(np.exp(qdeg[u] * (ld - top))))
    log_total -= len(q.src) * np.log(2.0 * n_edges)
    return float(np.exp(log_total) * len(q.src) * n_updates / n_edges)


def sample_cycle4(adj: Adjacency, vlab: np.ndarray, rng: np.random.Generator) -> QueryGraph:
    """A 4-cycle query whose labels are those of a random 4-cycle of the data graph."""
    n = len(adj.off) - 1
    deg = np.diff(adj.off)
    starts = np.nonzero(deg >= 2)[0]
    for _ in range(100000):
        a = int(rng.choice(starts))
        nb = adj.nbrs(a)
        b, d = [int(x) for x in rng.choice(nb, 2, replace=False)]
        common = np.intersect1d(adj.nbrs(b), adj.nbrs(d))
        common = common[common != a]
        if len(common) == 0:
            continue
        c = int(common[rng.integers(len(common))])
        vs = [a, b, c, d]
        el = [adj.edge_label(a, b), adj.edge_label(b, c), adj.edge_label(c, d), adj.edge_label(d, a)]
        return QueryGraph(np.array([vlab[v] for v in vs], dtype=np.uint32), np.array([0, 1, 2, 3], dtype=np.uint32),
                          np.array([1, 2, 3, 0], dtype=np.uint32), np.array(el, dtype=np.uint32))
    raise RuntimeError("no 4-cycle found")


@dataclass
class Workload:
    name: str
    data: DataGraph
    batches: List[Batch]
    queries: List[QueryGraph]
    batch_size: int
    meta: dict = field(default_factory=dict)


def loguniform_cuts(total: int, lo: int, hi: int, seed: int) -> List[int]:
    """Batch boundaries for `total` updates with sizes drawn log-uniformly from [lo, hi]."""
    rng = np.random.default_rng(seed)
    cuts, at = [0], 0
    while at < total:
        at = min(total, at + int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
        cuts.append(at)
    return cuts


def make_stream(n: int, s: np.ndarray, d: np.ndarray, el: np.ndarray, rng: np.random.Generator, n_ins: int,
                n_del: int, batch: int, holdout: float = 0.1, cuts: Optional[List[int]] = None):
    """Splits the edges into an initial graph and a held-out pool; the stream inserts n_ins pool
    edges and deletes n_del initial edges, randomly interleaved, cut into batches of `batch`
    updates (or at the given boundaries)."""
    m = len(s)
    perm = rng.permutation(m)
    nh = int(round(m * holdout))
    pool, init = perm[:nh], perm[nh:]
    if n_ins > len(pool):
        raise ValueError("not enough held-out edges")
    ins = pool[:n_ins]
    dels = rng.choice(init, size=n_del, replace=False) if n_del else np.zeros(0, dtype=np.int64)
    ops = np.concatenate([ins, dels])
    isdel = np.concatenate([np.zeros(len(ins), dtype=np.uint8), np.ones(len(dels), dtype=np.uint8)])
    order = rng.permutation(len(ops))
    ops, isdel = ops[order], isdel[order]
    # Orient each update edge at random (undirected edges, either endpoint first).
    flip = rng.random(len(ops)) < 0.5
    us = np.where(flip, d[ops], s[ops]).astype(np.uint32)
    vs = np.where(flip, s[ops], d[ops]).astype(np.uint32)
    batches = []
    if cuts is None:
        cuts = list(range(0, len(ops), batch)) + [len(ops)]
    for b0, b1 in zip(cuts[:-1], cuts[1:]):
        sl = slice(b0, b1)
        batches.append(Batch(us[sl], vs[sl], el[ops[sl]].astype(np.uint32), isdel[sl] if n_del else None))
    data = DataGraph(None, s[init], d[init], el[init])
    return data, batches


CONFIGS = {
    # Plain method, small size (4 uniform labels, 5k insertions, batch 1024, 4-cycle).
    "c1": dict(n=10_000, m=50_000, gamma=2.3, nvl=4, vzipf=None, nel=1, ezipf=None, cap=False, n_ins=5_000, n_del=0,
               batch=1024, queries=[("cycle4", 4)]),
    # Amazon-shaped: 400k vertices, 2.4M edges, 6 Zipf(1.0) labels, 240k updates (10% deletions).
    "c2": dict(n=400_000, m=2_400_000, gamma=2.1, nvl=6, vzipf=1.0, nel=1, ezipf=None, cap=True, n_ins=216_000,
               n_del=24_000, batch=65_536, queries=[("dense", 6)] * 5 + [("tree", 6)] * 5),
    # LiveJournal-shaped heavy-vertex stress: 4.8M vertices, 43M edges, 20 Zipf(1.2) labels.
    # Dense 8-vertex queries over all labels have 1e11-1e15 new matches per 1M-update batch
    # (more than any engine enumerates in seconds), so they are sampled from the subgraph of
    # the 12 rarest labels (query_min_label: labels are numbered by frequency rank) and a
    # candidate is kept only when its expected_batch_matches is at most query_bound; candidate
    # t of query i uses seed + i + 1000 t.
    "c3": dict(n=4_800_000, m=43_000_000, gamma=1.9, nvl=20, vzipf=1.2, nel=1, ezipf=None, cap=True,
               n_ins=2_150_000, n_del=2_150_000, batch=1_000_000, queries=[("dense", 8)] * 4,
               query_min_label=8, query_bound=2e15),
    # Batched multi-query: the Amazon-shaped graph, 64 queries of 4..12 vertices, dense and sparse.
    "c4": dict(n=400_000, m=2_400_000, gamma=2.1, nvl=6, vzipf=1.0, nel=1, ezipf=None, cap=True, n_ins=216_000,
               n_del=24_000, batch=65_536, queries="mixed64"),
    # Serving: Netflow-shaped multi-label graph, 32 queries of 4..10 vertices.
    # 32 queries of 4..10 vertices, dense and sparse.  Batch sizes are log-uniform in
    # [1k, 256k] (batch_range); `batch` is the largest.
    "c5": dict(n=3_000_000, m=20_000_000, gamma=2.1, nvl=8, vzipf=None, nel=16, ezipf=1.1, cap=True,
               n_ins=700_000, n_del=300_000, batch=262_144, batch_range=(1_024, 262_144), queries="mixed32"),
}


def scaled(name: str, scale: float) -> dict:
    """A configuration with vertex/edge/update counts multiplied by `scale` (for tests)."""
    c = dict(CONFIGS[name])
    for k in ("n", "m", "n_ins", "n_del", "batch"):
        c[k] = max(1, int(c[k] * scale))
    return c


def make_workload(name: str, cfg: Optional[dict] = None, seed: Optional[int] = None, nqueries: Optional[int] = None) -> Workload:
    cfg = dict(CONFIGS[name] if cfg is None else cfg)
    index = int(name[1:]) if name[1:].isdigit() else 0
    seed = 1000 + index if seed is None else seed
    rng = np.random.default_rng(seed)
    s, d = chung_lu(cfg["n"], cfg["m"], cfg["gamma"], rng, cap=cfg["cap"])
    vlab = draw_labels(cfg["n"], cfg["nvl"], rng, cfg["vzipf"])
    el = draw_labels(len(s), cfg["nel"], rng, cfg["ezipf"]) if cfg["nel"] > 1 else np.zeros(len(s), dtype=np.uint32)
    cuts = None
    if cfg.get("batch_range"):
        lo, hi = cfg["batch_range"]
        hi = min(hi, cfg["batch"])
        cuts = loguniform_cuts(cfg["n_ins"] + cfg["n_del"], min(lo, hi), hi, seed + 7919)
    data, batches = make_stream(cfg["n"], s, d, el, rng, cfg["n_ins"], cfg["n_del"], cfg["batch"], cuts=cuts)
    data.vlabels = vlab
    adj = Adjacency(cfg["n"], data.src, data.dst, data.elabels)
    qspec = cfg["queries"]
    if qspec == "mixed64" or qspec == "mixed32":
        nq, kmax = (64, 12) if qspec == "mixed64" else (32, 10)
        qspec = [("dense" if i % 2 == 0 else "sparse", int(np.random.default_rng(seed + i).integers(4, kmax + 1)))
                 for i in range(nq)]
    if nqueries is not None:
        qspec = qspec[:nqueries]
    queries = []
    lmin, bound = cfg.get("query_min_label"), cfg.get("query_bound")
    qadj = adj
    if lmin is not None:
        keep = (vlab[data.src] >= lmin) & (vlab[data.dst] >= lmin)
        qadj = Adjacency(cfg["n"], data.src[keep], data.dst[keep], data.elabels[keep])
    deg = np.diff(adj.off) if bound is not None else None
    for i, (kind, k) in enumerate(qspec):
        if kind == "cycle4":
            queries.append(sample_cycle4(adj, vlab, np.random.default_rng(seed + i)))
            continue
        if bound is None:
            queries.append(sample_query(qadj, vlab, k, kind, np.random.default_rng(seed + i)))
            continue
        best, best_est = None, None
        for t in range(200):
            q = sample_query(qadj, vlab, k, kind, np.random.default_rng(seed + i + 1000 * t))
            est = expected_batch_matches(q, vlab, deg, len(data.src), cfg["batch"])
            if best is None or est < best_est:
                best, best_est = q, est
            if est <= bound:
                break
        queries.append(best)
    return Workload(name, data, batches, queries, cfg["batch"], meta=cfg)
