"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle, batch by batch.

Counts are integers and must be bit-exact: positive and negative incremental matches per
batch and per query, the per-query-edge split, and (with materialisation) the sorted rows.
"""
import numpy as np
import pytest

import csm
from csm import Batch, DataGraph, QueryGraph, gen
from oracle import Oracle
from helpers import clique, cycle, path, random_graph, small_workload, star

pytestmark = pytest.mark.gpu


def check_stream(w, queries=None, batches=None, rows=False, stats=None, **cfg):
    queries = w.queries if queries is None else queries
    batches = w.batches if batches is None else batches
    if rows:
        cfg.setdefault("materialize_rows", 1 << 22)
    eng = csm.Engine(**cfg)
    for q in queries:
        eng.load_query(q)
    eng.load_graph(w.data)
    oracles = [Oracle(q, w.data) for q in queries]
    totals = [0, 0]
    for bi, b in enumerate(batches):
        res = eng.apply(b)
        for qi, o in enumerate(oracles):
            r = o.apply(b, rows=rows)
            got = (res[qi].positive, res[qi].negative)
            assert got == (r["pos"], r["neg"]), f"batch {bi} query {qi}: engine {got} oracle {(r['pos'], r['neg'])}"
            pos, neg = eng.edge_counts(qi)
            assert pos == r["per_qe_pos"] and neg == r["per_qe_neg"], f"batch {bi} query {qi} per-edge split"
            if rows:
                assert np.array_equal(eng.embeddings(qi, 1), o.rows(1)), f"batch {bi} query {qi} positive rows"
                assert np.array_equal(eng.embeddings(qi, -1), o.rows(-1)), f"batch {bi} query {qi} negative rows"
            totals[0] += r["pos"]
            totals[1] += r["neg"]
    if stats is not None:
        stats.append(eng.stats())
    eng.close()
    return totals


@pytest.fixture(scope="module")
def c1():
    return small_workload("c1")


@pytest.mark.parametrize("strategy", [0, 1, 2, 3])
def test_c1_search_strategies(c1, strategy):
    tot = check_stream(c1, algorithm=0, search_strategy=strategy)
    assert tot[0] > 0


@pytest.mark.parametrize("algorithm", [1, 2, 4, 5])
def test_c1_algorithm_presets(c1, algorithm):
    check_stream(c1, algorithm=algorithm)


@pytest.mark.parametrize("order", [0, 1, 2, 3])
def test_c1_matching_orders_no_cartesian(c1, order):
    check_stream(c1, algorithm=0, matching_order=order, cartesian_product=0)


def test_c1_rows(c1):
    w = small_workload("c1", scale=0.3)
    check_stream(w, rows=True)


def test_amazon_shaped_small_with_deletions():
    w = small_workload("c2", scale=0.005, batch=700, nqueries=6)
    tot = check_stream(w, search_strategy=2)
    assert tot[1] > 0


def test_amazon_shaped_small_dfs_with_stealing():
    w = small_workload("c2", scale=0.005, batch=1500, nqueries=6)
    check_stream(w, search_strategy=0)


def test_rows_with_deletions():
    w = small_workload("c2", scale=0.002, batch=300, nqueries=3)
    check_stream(w, rows=True)


def test_multi_query_mixed_sizes():
    w = small_workload("c4", scale=0.002, batch=500, nqueries=6)
    check_stream(w)


def test_heavy_vertex_dense8():
    w = small_workload("c3", scale=0.0005, batch=2000, nqueries=2)
    check_stream(w)


def query_graph(labels, edges):
    s, d = zip(*edges)
    return QueryGraph(np.asarray(labels, dtype=np.uint32), np.array(s, dtype=np.uint32), np.array(d, dtype=np.uint32),
                      np.zeros(len(edges), dtype=np.uint32))


K23 = [(0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (1, 4)]
HOUSE = [(0, 1), (1, 2), (2, 3), (3, 0), (0, 4), (1, 4)]
LADDER = [(0, 1), (1, 2), (3, 4), (4, 5), (0, 3), (1, 4), (2, 5)]


@pytest.mark.parametrize("strategy", [0, 1, 2, 3])
@pytest.mark.parametrize("order", [0, 1])
def test_last_level_shared_by_the_level_above(strategy, order):
    """Plans whose last query vertex is not adjacent to the vertex matched before it count the
    last level once per prefix and subtract, per vertex above, whether that vertex is itself a
    candidate (injectivity): same labels (the subtraction applies) and distinct labels (it
    cannot), with deletions, under every search strategy."""
    rng = np.random.default_rng(11)
    n = 1500
    vl, s, d, el = random_graph(n, 15000, 2, rng)
    data, batches = gen.make_stream(n, s, d, el, rng, n_ins=1200, n_del=300, batch=500)
    data = DataGraph(vl, data.src, data.dst, data.elabels)
    queries = [query_graph([0] * 5, K23), query_graph([0, 0, 1, 1, 1], K23),
               query_graph([0, 1, 0, 1, 1], HOUSE), query_graph([0] * 6, LADDER)]
    w = gen.Workload("shared-last", data, batches, queries, 500)
    st = []
    tot = check_stream(w, stats=st, search_strategy=strategy, matching_order=order)
    assert tot[0] > 0 and tot[1] > 0
    assert st[0].enum_shared_last > 0


PENDANT = [(2, 3), (2, 4), (2, 5), (3, 4), (3, 5), (4, 5), (1, 2), (0, 1)]


@pytest.mark.parametrize("strategy", [0, 1, 2, 3])
def test_pendant_counting_level(strategy):
    """A 4-clique with a two-vertex path hanging off it, the path's label absent from the clique:
    plans that start inside the clique count the path from per-vertex tables filled each phase
    (the table kernel, the settling of sibling buffers, and the donation and expansion limits)."""
    rng = np.random.default_rng(5)
    n = 1200
    vl, s, d, el = random_graph(n, 16000, 3, rng)
    data, batches = gen.make_stream(n, s, d, el, rng, n_ins=1200, n_del=300, batch=500)
    data = DataGraph(vl, data.src, data.dst, data.elabels)
    queries = [query_graph([0, 0, 1, 2, 1, 2], PENDANT), query_graph([2, 0, 1, 1, 1, 1], PENDANT)]
    w = gen.Workload("pendant", data, batches, queries, 500)
    with csm.Engine(search_strategy=strategy) as eng:
        eng.load_query(queries[0])
        eng.load_graph(data)
        assert eng.describe(0).count("pendant counting level") > 0
    tot = check_stream(w, search_strategy=strategy)
    assert tot[0] > 0 and tot[1] > 0


def test_edge_cases_in_batches():
    rng = np.random.default_rng(7)
    vl, s, d, el = random_graph(60, 300, 2, rng)
    data = DataGraph(vl, s, d, el)
    w = gen.Workload("edge", data, [], [cycle(4, [0, 1, 0, 1]), clique(3), star(3), path(4)], 0)
    n = len(vl)
    batches = [
        Batch(np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32)),         # empty
        Batch(s[:5], d[:5], el[:5]),                                                           # existing edges
        Batch(np.array([3, 3, 5, 5], np.uint32), np.array([3, 9, 9, 3], np.uint32),
              np.zeros(4, np.uint32)),                                                         # self-loop + dups
        Batch(np.array([1, 2, n + 5], np.uint32), np.array([40, 41, 2], np.uint32),
              np.zeros(3, np.uint32), np.array([1, 1, 0], np.uint8)),                          # absent deletes, out of range
        Batch(s[10:20], d[10:20], el[10:20], np.ones(10, np.uint8)),                           # deletions
        Batch(np.concatenate([s[10:15], s[30:35]]), np.concatenate([d[10:15], d[30:35]]),
              np.concatenate([el[10:15], el[30:35]]),
              np.array([0] * 5 + [1] * 5, np.uint8)),                                           # re-insert + delete
        Batch(np.array([7, 7], np.uint32), np.array([8, 8], np.uint32), np.zeros(2, np.uint32),
              np.array([1, 0], np.uint8)),                                                      # insert wins
    ]
    for strategy in (0, 2):
        check_stream(w, batches=batches, search_strategy=strategy)


@pytest.mark.parametrize("bs", [1, 13])
def test_tiny_batches(bs):
    w = small_workload("c1", scale=0.05)
    xs = np.concatenate([b.src for b in w.batches])[:300]
    ys = np.concatenate([b.dst for b in w.batches])[:300]
    ls = np.concatenate([b.elabels for b in w.batches])[:300]
    batches = [Batch(xs[i:i + bs], ys[i:i + bs], ls[i:i + bs]) for i in range(0, len(xs), bs)][:60]
    check_stream(w, batches=batches)


def test_pool_regrowth_keeps_counts():
    w = small_workload("c2", scale=0.005, batch=2000, nqueries=3)
    # A pool barely larger than the initial layout forces relocation, overflow and regrowth.
    eng = csm.Engine()
    for q in w.queries:
        eng.load_query(q)
    eng.load_graph(w.data)
    used = eng.stats().pool_used
    eng.close()
    tot = check_stream(w, pool_entries=int(used * 1.05) + 64)
    assert tot[0] > 0


def test_launch_shapes_and_steal_chunk():
    w = small_workload("c2", scale=0.003, batch=3000, nqueries=4)
    for bps, wpb, sc in ((1, 1, 32), (2, 4, 128), (8, 8, 64)):
        check_stream(w, blocks_per_sm=bps, warps_per_block=wpb, steal_chunk=sc, search_strategy=0)


def test_autotune_keeps_counts_and_reports_choice():
    # Tuning re-runs the insertion phase under each candidate configuration; the counts of
    # the tuned batches and of the batches after them must not change.
    w = small_workload("c2", scale=0.003, batch=3000, nqueries=3)
    check_stream(w, search_strategy=2, autotune_batches=2)
    eng = csm.Engine(search_strategy=2, autotune_batches=2)
    eng.load_query(w.queries[0])
    eng.load_graph(w.data)
    for b in w.batches[:3]:
        eng.apply(b)
    st = eng.stats()
    assert st.tuned_strategy in (0, 2, 3)
    assert st.tuned_steal_chunk in (8, 64)
    assert st.tuned_warps_per_block in (4, 8)
    assert st.tuned_occupancy in (4, 6)
    eng.close()


@pytest.mark.parametrize("strategy", [0, 1])
def test_cuda_graph_replay_matches_oracle(strategy):
    # Batches of two sizes (one capture each, then replays), with deletions.
    w = small_workload("c2", scale=0.003, batch=1500, nqueries=4)
    check_stream(w, search_strategy=strategy, cuda_graphs=1)
    eng = csm.Engine(search_strategy=strategy, cuda_graphs=1)
    eng.load_query(w.queries[0])
    eng.load_graph(w.data)
    for b in w.batches:
        eng.apply(b)
    assert eng.stats().graph_launches >= len(w.batches) - 1
    eng.close()


def test_cuda_graph_device_updates_and_autotune():
    import torch
    w = small_workload("c2", scale=0.003, batch=1500, nqueries=3)
    ref = csm.Engine(search_strategy=0)
    eng = csm.Engine(search_strategy=0, cuda_graphs=1, autotune_batches=1)
    for e in (ref, eng):
        for q in w.queries:
            e.load_query(q)
        e.load_graph(w.data)
    for b in list(w.batches) * 2:
        want = [(r.positive, r.negative) for r in ref.apply(b)]
        dl = b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
        arrs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in
                (b.src.astype(np.int32), b.dst.astype(np.int32), b.elabels.astype(np.int32), dl.astype(np.uint8))]
        got = eng.apply_device(len(b.src), *[a.data_ptr() for a in arrs])
        assert [(r.positive, r.negative) for r in got] == want
    ref.close()
    eng.close()


@pytest.mark.parametrize("graphs", [0, 1])
def test_live_replanning_keeps_counts(graphs):
    # A 1% drift threshold re-plans after nearly every batch; the counts must not change.
    w = small_workload("c2", scale=0.003, batch=1500, nqueries=4)
    check_stream(w, replan_drift_pct=1, cuda_graphs=graphs, search_strategy=0 if graphs else 2)
    eng = csm.Engine(replan_drift_pct=1)
    for q in w.queries:
        eng.load_query(q)
    eng.load_graph(w.data)
    for b in w.batches:
        eng.apply(b)
    assert eng.stats().replans >= 1
    eng.close()


def test_snapshot_restore_continues_stream(tmp_path):
    w = small_workload("c2", scale=0.003, batch=1500, nqueries=3)
    a = csm.Engine()
    for q in w.queries:
        a.load_query(q)
    a.load_graph(w.data)
    half = len(w.batches) // 2
    for b in w.batches[:half]:
        a.apply(b)
    snap = str(tmp_path / "state.snap")
    a.save_snapshot(snap)
    b_eng = csm.Engine(search_strategy=0)
    for q in w.queries:
        b_eng.load_query(q)
    b_eng.load_snapshot(snap)
    oracles = [Oracle(q, w.data) for q in w.queries]
    for bt in w.batches[:half]:
        for o in oracles:
            o.apply(bt)
    for bt in w.batches[half:]:
        ra = [(r.positive, r.negative) for r in a.apply(bt)]
        rb = [(r.positive, r.negative) for r in b_eng.apply(bt)]
        ro = [(x["pos"], x["neg"]) for x in (o.apply(bt) for o in oracles)]
        assert ra == rb == ro
    # A snapshot is refused by an engine with other queries.
    c = csm.Engine()
    c.load_query(w.queries[0])
    with pytest.raises(csm.CsmError):
        c.load_snapshot(snap)
    for e in (a, b_eng, c):
        e.close()


def test_work_counters_do_not_depend_on_the_schedule():
    """The roofline's algorithmic bytes come from the kernel's work counters (pivot entries
    scanned, membership probes, tail lists): per expanded partial embedding, never per launch or
    per warp, so they are the same under every search strategy, launch shape and donation
    granularity for the same batches."""
    w = small_workload("c2", scale=0.01, batch=1500, nqueries=6)
    seen = {}
    for cfg in (dict(search_strategy=0), dict(search_strategy=1), dict(search_strategy=2),
                dict(search_strategy=3), dict(search_strategy=0, warps_per_block=4, steal_chunk=8),
                dict(search_strategy=2, semi_bfs_items_per_warp=8)):
        with csm.Engine(**cfg) as eng:
            for q in w.queries:
                eng.load_query(q)
            eng.load_graph(w.data)
            counts = [[(r.positive, r.negative) for r in eng.apply(b)] for b in w.batches[:3]]
            st = eng.stats()
            seen[str(cfg)] = (counts, st.enum_scan_entries, st.enum_probes, st.enum_tail_lists)
    first = next(iter(seen.values()))
    assert first[1] > 0 and first[2] > 0
    for k, v in seen.items():
        assert v == first, k
