"""GPU tests of the enumeration's work-donation ring and its time limit.

* A ring of 32 slots fills at once; a full ring may only cost balance, never a result: counts
  must still equal the oracle's, with donations refused.
* The same batch applied again and again from one restored state must count the same matches
  every time, at a size where launches donate heavily.
* A launch that runs past its time limit stops early: the call reports CSM_ERR_TIMEOUT, the
  batch is still applied to the graph in full, and the next batch counts exactly.
"""
import os

import numpy as np
import pytest

import csm
from csm import Batch
from helpers import small_workload
from oracle import Oracle

pytestmark = pytest.mark.gpu


def inverse(b):
    dl = b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
    return Batch(b.src, b.dst, b.elabels, (1 - dl).astype(np.uint8))


@pytest.mark.parametrize("strategy", [0, 2])
def test_tiny_donation_ring_equals_oracle(strategy):
    w = small_workload("c2", scale=0.005, batch=700, nqueries=6)
    eng = csm.Engine(search_strategy=strategy, queue_slots=32, steal_chunk=8)
    for q in w.queries:
        eng.load_query(q)
    eng.load_graph(w.data)
    oracles = [Oracle(q, w.data) for q in w.queries]
    for bi, b in enumerate(w.batches):
        res = eng.apply(b)
        for qi, o in enumerate(oracles):
            r = o.apply(b)
            assert (res[qi].positive, res[qi].negative) == (r["pos"], r["neg"]), f"batch {bi} query {qi}"
    st = eng.stats()
    eng.close()
    if strategy == 0:
        assert st.donations > 0


def test_queue_slots_validated():
    with pytest.raises(csm.CsmError) as ei:
        csm.Engine(queue_slots=48)
    assert ei.value.code == -1
    with pytest.raises(csm.CsmError):
        csm.Engine(queue_slots=16)


def test_replayed_batch_counts_are_stable(tmp_path):
    """One dense-query batch of the Amazon-shaped graph at 20% scale, applied five times from the
    same state (undone by its inverse in between, and once restored from a snapshot)."""
    w = small_workload("c2", scale=0.2, nqueries=5)
    q = w.queries[0]
    eng = csm.Engine(search_strategy=2, steal_chunk=16)
    eng.load_query(q)
    eng.load_graph(w.data)
    eng.apply(w.batches[0])
    snap = str(tmp_path / "state.snap")
    eng.save_snapshot(snap)
    b, undo = w.batches[1], inverse(w.batches[1])
    counts = []
    for _ in range(4):
        r = eng.apply(b)[0]
        counts.append((r.positive, r.negative))
        eng.apply(undo)
    st = eng.stats()
    eng.close()
    eng2 = csm.Engine(search_strategy=0, steal_chunk=16, queue_slots=1024)
    eng2.load_query(q)
    eng2.load_snapshot(snap)
    r = eng2.apply(b)[0]
    counts.append((r.positive, r.negative))
    eng2.close()
    assert counts[0][0] > 0
    assert len(set(counts)) == 1, counts
    assert st.donations > 0


def test_time_limit_stops_launch_and_keeps_graph_consistent():
    w = small_workload("c2", scale=0.05, nqueries=2)
    ref = csm.Engine(search_strategy=2)
    lim = csm.Engine(search_strategy=2, time_limit_us=1)
    for e in (ref, lim):
        for q in w.queries:
            e.load_query(q)
        e.load_graph(w.data)
    full = ref.apply(w.batches[0])
    rc, part = lim.apply_partial(w.batches[0])
    assert rc == -4, "a 1-microsecond limit must stop the launch"
    assert "time limit" in lim._err(lim._h)
    for qi in range(len(w.queries)):
        assert part[qi].positive <= full[qi].positive and part[qi].negative <= full[qi].negative
        assert (part[qi].inserted, part[qi].deleted) == (full[qi].inserted, full[qi].deleted)
    assert sum(r.positive for r in part) < sum(r.positive for r in full)
    # The graph holds the whole batch: with the limit lifted, later batches count exactly.
    lim.set_time_limit(0)
    for b in w.batches[1:3]:
        a, c = ref.apply(b), lim.apply(b)
        assert [(r.positive, r.negative) for r in a] == [(r.positive, r.negative) for r in c]
    ref.close()
    lim.close()


def test_time_limit_on_depth_first_and_oracle_after():
    """Depth-first launch with donation, stopped by its limit; the next batches equal the oracle."""
    w = small_workload("c2", scale=0.02, nqueries=3)
    eng = csm.Engine(search_strategy=0, time_limit_us=1)
    for q in w.queries:
        eng.load_query(q)
    eng.load_graph(w.data)
    oracles = [Oracle(q, w.data) for q in w.queries]
    rc, _ = eng.apply_partial(w.batches[0])
    for o in oracles:
        o.apply(w.batches[0])
    eng.set_time_limit(0)
    for b in w.batches[1:]:
        res = eng.apply(b)
        for qi, o in enumerate(oracles):
            r = o.apply(b)
            assert (res[qi].positive, res[qi].negative) == (r["pos"], r["neg"])
    eng.close()
    assert rc in (0, -4)
