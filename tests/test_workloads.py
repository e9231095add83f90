"""CPU tests of the synthetic workloads (gcsm-bu_b200/csm/gen.py) and the properties the bench
relies on: every stream update is effective (inserts absent edges, deletes present ones), so
applying a batch's inverse right after it restores the graph; batch-size ranges; query shapes."""
import numpy as np
import pytest

from csm import gen


def edge_set(src, dst):
    return {(min(int(a), int(b)), max(int(a), int(b))) for a, b in zip(src, dst)}


@pytest.mark.parametrize("name,scale", [("c2", 0.01), ("c5", 0.005), ("c4", 0.01)])
def test_stream_updates_are_all_effective(name, scale):
    w = gen.make_workload(name, gen.scaled(name, scale), nqueries=2)
    present = edge_set(w.data.src, w.data.dst)
    for b in w.batches:
        dl = b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
        for x, y, d in zip(b.src, b.dst, dl):
            e = (min(int(x), int(y)), max(int(x), int(y)))
            if d:
                assert e in present, "deletion of an absent edge"
                present.remove(e)
            else:
                assert e not in present, "insertion of a present edge"
                present.add(e)


def test_loguniform_batch_sizes():
    cuts = gen.loguniform_cuts(1_000_000, 1_024, 262_144, seed=5)
    sizes = np.diff(cuts)
    assert cuts[0] == 0 and cuts[-1] == 1_000_000
    assert (sizes[:-1] >= 1_024).all() and (sizes <= 262_144).all()
    assert len(set(sizes.tolist())) > len(sizes) // 2  # sizes vary


def connected(nv, src, dst):
    adj = {v: set() for v in range(nv)}
    for a, b in zip(src, dst):
        adj[int(a)].add(int(b))
        adj[int(b)].add(int(a))
    seen, stack = {0}, [0]
    while stack:
        for u in adj[stack.pop()]:
            if u not in seen:
                seen.add(u)
                stack.append(u)
    return len(seen) == nv


def test_query_shapes():
    w = gen.make_workload("c4", gen.scaled("c4", 0.01))
    assert len(w.queries) == 64
    for i, q in enumerate(w.queries):
        k, m = q.nv, len(q.src)
        assert 4 <= k <= 12 and connected(k, q.src, q.dst)
        assert len(edge_set(q.src, q.dst)) == m  # no duplicate edges
        if i % 2 == 1:  # sparse: at least one cycle, average degree below 3
            assert k <= m and 2 * m < 3 * k
    w2 = gen.make_workload("c2", gen.scaled("c2", 0.01))
    for q in w2.queries[5:]:  # trees
        assert len(q.src) == q.nv - 1 and connected(q.nv, q.src, q.dst)
