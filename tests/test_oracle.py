"""CPU tests of the oracle: closed forms, the |M(G')| - |M(G)| identity, batch-split invariance."""
import numpy as np
import pytest

from csm import Batch, DataGraph, QueryGraph, gen
from oracle import Oracle
from helpers import clique, cycle, path, random_graph, star


def complete_graph(n, missing=()):
    es = [(i, j) for i in range(n) for j in range(i + 1, n) if (i, j) not in missing]
    s, d = zip(*es)
    return DataGraph(np.zeros(n, dtype=np.uint32), np.array(s, dtype=np.uint32), np.array(d, dtype=np.uint32),
                     np.zeros(len(s), dtype=np.uint32))


def one(x, y, dele=False):
    return Batch(np.array([x], dtype=np.uint32), np.array([y], dtype=np.uint32), np.zeros(1, dtype=np.uint32),
                 np.array([1], dtype=np.uint8) if dele else None)


@pytest.mark.parametrize("n", [4, 5, 7])
def test_triangle_in_clique_insert_and_delete(n):
    o = Oracle(clique(3), complete_graph(n, missing={(0, 1)}))
    assert o.count_all() == n * (n - 1) * (n - 2) - 6 * (n - 2)
    r = o.apply(one(1, 0))
    assert r["pos"] == 6 * (n - 2) and r["neg"] == 0
    assert o.count_all() == n * (n - 1) * (n - 2)
    r = o.apply(one(0, 1, dele=True))
    assert r["neg"] == 6 * (n - 2) and r["pos"] == 0


@pytest.mark.parametrize("k,deg", [(2, 5), (3, 6), (4, 4)])
def test_star_falling_factorial(k, deg):
    # Data: a star with `deg` leaves; the query star with k leaves maps its centre to the hub.
    data = DataGraph(np.zeros(deg + 2, dtype=np.uint32), np.zeros(deg, dtype=np.uint32),
                     np.arange(1, deg + 1, dtype=np.uint32), np.zeros(deg, dtype=np.uint32))
    o = Oracle(star(k), data)
    ff = lambda d: int(np.prod([d - i for i in range(k)])) if d >= k else 0
    assert o.count_all() == ff(deg) + (ff(1) if k == 1 else 0)
    r = o.apply(one(0, deg + 1))
    assert r["pos"] == ff(deg + 1) - ff(deg)


def test_cycle4_closed_form():
    # K4 has 3 distinct 4-cycles, 8 automorphic images each.
    o = Oracle(cycle(4), complete_graph(4))
    assert o.count_all() == 24
    # Deleting one edge of K4 destroys the 2 cycles through it.
    r = o.apply(one(0, 1, dele=True))
    assert r["neg"] == 16 and o.count_all() == 8


def test_labels_must_match():
    q = QueryGraph(np.array([1, 2], dtype=np.uint32), np.array([0], dtype=np.uint32), np.array([1], dtype=np.uint32),
                   np.array([7], dtype=np.uint32))
    data = DataGraph(np.array([1, 2, 1], dtype=np.uint32), np.array([0], dtype=np.uint32), np.array([1], dtype=np.uint32),
                     np.array([7], dtype=np.uint32))
    o = Oracle(q, data)
    assert o.count_all() == 1
    b = Batch(np.array([2, 2], dtype=np.uint32), np.array([1, 0], dtype=np.uint32), np.array([7, 7], dtype=np.uint32))
    assert o.apply(b)["pos"] == 1  # (2,1) matches, (2,0) has two label-1 endpoints


@pytest.mark.parametrize("seed", range(6))
def test_delta_identity_random(seed):
    rng = np.random.default_rng(seed)
    vl, s, d, el = random_graph(40, 160, 2, rng, nel=2)
    data = DataGraph(vl, s, d, el)
    adj = gen.Adjacency(40, s, d, el)
    q = gen.sample_query(adj, vl, 4 + seed % 2, "dense" if seed % 2 else "tree", rng)
    o = Oracle(q, data)
    for _ in range(3):
        before = o.count_all()
        nb = 30
        x = rng.integers(0, 40, nb).astype(np.uint32)
        y = rng.integers(0, 40, nb).astype(np.uint32)
        b = Batch(x, y, rng.integers(0, 2, nb).astype(np.uint32), (rng.random(nb) < 0.4).astype(np.uint8))
        r = o.apply(b, threads=3)
        assert sum(r["per_qe_pos"]) == r["pos"] and sum(r["per_qe_neg"]) == r["neg"]
        assert o.count_all() - before == r["pos"] - r["neg"]


def test_batch_split_invariance():
    w = gen.make_workload("c1", gen.scaled("c1", 0.3))
    totals = []
    for bs in (50, 400, 1500):
        o = Oracle(w.queries[0], w.data)
        stream = [b for b in w.batches]
        xs = np.concatenate([b.src for b in stream])
        ys = np.concatenate([b.dst for b in stream])
        ls = np.concatenate([b.elabels for b in stream])
        tot = 0
        for b0 in range(0, len(xs), bs):
            tot += o.apply(Batch(xs[b0:b0 + bs], ys[b0:b0 + bs], ls[b0:b0 + bs]))["pos"]
        totals.append(tot)
    assert len(set(totals)) == 1 and totals[0] > 0


def test_rows_sorted_unique_and_counted():
    w = gen.make_workload("c1", gen.scaled("c1", 0.2))
    o = Oracle(w.queries[0], w.data)
    r = o.apply(w.batches[0], rows=True)
    rows = o.rows(1)
    assert len(rows) == r["pos"]
    as_tuples = [tuple(x) for x in rows]
    assert as_tuples == sorted(as_tuples) and len(set(as_tuples)) == len(as_tuples)
    for row in rows:
        assert len(set(row)) == len(row)  # injective


def brute_embeddings(q, vlab, edges):
    """All embeddings of query q (vertex-id order rows) in a small labelled graph given as a
    set of (min, max, label) edges (one vertex pair may carry edges of several labels, each its
    own edge, as in the label-partitioned relations), by exhaustive search over injective maps."""
    import itertools
    nv = len(q.vlabels)
    qe = list(zip(q.src.tolist(), q.dst.tolist(), q.elabels.tolist()))
    out = set()
    cands = [[v for v in range(len(vlab)) if vlab[v] == q.vlabels[u]] for u in range(nv)]
    for f in itertools.product(*cands):
        if len(set(f)) != nv:
            continue
        if all((min(f[a], f[b]), max(f[a], f[b]), l) in edges for a, b, l in qe):
            out.add(tuple(int(x) for x in f))
    return out


@pytest.mark.parametrize("seed", range(24))
def test_positive_and_negative_rows_against_brute_force(seed):
    # Independent of any decomposition rule: the positive rows of a batch are exactly the
    # embeddings of the graph after it that were not embeddings before, the negative rows those
    # that disappeared; with repeated updates, both orientations and insert+delete of one edge.
    rng = np.random.default_rng(100 + seed)
    n = 9
    vl, s, d, el = random_graph(n, 16, 2, rng, nel=2)
    data = DataGraph(vl, s, d, el)
    edges = {(min(int(a), int(b)), max(int(a), int(b)), int(l)) for a, b, l in zip(s, d, el)}
    adj = gen.Adjacency(n, s, d, el)
    kind = ["tree", "dense", "sparse"][seed % 3]
    q = gen.sample_query(adj, vl, 3 + seed % 2, kind, rng)
    o = Oracle(q, data)
    for _ in range(3):
        nb = 8
        x = rng.integers(0, n, nb).astype(np.uint32)
        y = rng.integers(0, n, nb).astype(np.uint32)
        lab = rng.integers(0, 2, nb).astype(np.uint32)
        dl = (rng.random(nb) < 0.4).astype(np.uint8)
        if seed % 2:  # repeat one update in the other orientation
            x[-1], y[-1], lab[-1], dl[-1] = y[0], x[0], lab[0], dl[0]
        before = brute_embeddings(q, vl, edges)
        # Set semantics of a batch: deletions of present edges, then insertions of absent ones
        # (an edge both inserted and deleted in one batch ends present); self-loops are ignored.
        dels = {(min(int(a), int(b)), max(int(a), int(b)), int(l)) for a, b, l, z in zip(x, y, lab, dl)
                if z and a != b}
        ins = {(min(int(a), int(b)), max(int(a), int(b)), int(l)) for a, b, l, z in zip(x, y, lab, dl)
               if not z and a != b}
        edges = (edges - dels) | ins
        after = brute_embeddings(q, vl, edges)
        r = o.apply(Batch(x, y, lab, dl), rows=True)
        pos_rows = {tuple(int(v) for v in row) for row in o.rows(1)}
        neg_rows = {tuple(int(v) for v in row) for row in o.rows(-1)}
        assert pos_rows == after - before and r["pos"] == len(after - before)
        assert neg_rows == before - after and r["neg"] == len(before - after)
