"""GPU tests of the serving loop (include/csm_server.h): every result of a request served in a
mix of tenants, slots and memory grants equals the result of the same tenant engine applying
the same batches alone through csm_apply_batch, and the alone results equal the CPU oracle."""
import numpy as np
import pytest

import csm
from oracle import Oracle
from helpers import small_workload

pytestmark = pytest.mark.gpu


def tenant_groups(w, sizes):
    groups, at = [], 0
    for k in sizes:
        groups.append(w.queries[at: at + k])
        at += k
    return groups


def make_engine(queries, data, **cfg):
    cfg.setdefault("frontier_bytes", 1 << 20)
    eng = csm.Engine(**cfg)
    for q in queries:
        eng.load_query(q)
    eng.load_graph(data)
    return eng


def alone(w, groups, batches, **cfg):
    out = []
    for g in groups:
        eng = make_engine(g, w.data, **cfg)
        out.append([[(r.positive, r.negative) for r in eng.apply(b)] for b in batches])
        eng.close()
    return out


def served(w, groups, batches, slots, budget, per_tenant=False, **cfg):
    engines = [make_engine(g, w.data, **cfg) for g in groups]
    srv = csm.Server(slots=slots, memory_budget=budget, min_frontier_bytes=1 << 16)
    for e in engines:
        srv.add_tenant(e)
    got = [[None] * len(batches) for _ in groups]
    if per_tenant:
        # Interleave single-tenant requests: batch b for tenant t, tenants in rotating order.
        ids = []
        for bi, b in enumerate(batches):
            for k in range(len(groups)):
                t = (bi + k) % len(groups)
                ids.append((t, bi, srv.submit(b, tenant=t)))
        for t, bi, rid in ids:
            info, res = srv.wait(rid)
            assert info.status == 0 and info.done_ns >= info.start_ns >= info.arrival_ns
            got[t][bi] = [(r.positive, r.negative) for r in res]
    else:
        ids = [srv.submit(b) for b in batches]
        for bi, rid in enumerate(ids):
            info, res = srv.wait(rid)
            assert info.status == 0
            at = 0
            for t, g in enumerate(groups):
                got[t][bi] = [(r.positive, r.negative) for r in res[at: at + len(g)]]
                at += len(g)
    st = srv.stats()
    srv.close()
    for e in engines:
        e.close()
    return got, st


@pytest.fixture(scope="module")
def wl():
    return small_workload("c2", scale=0.004, batch=300, nqueries=6)


def test_alone_matches_oracle(wl):
    groups = tenant_groups(wl, [2, 3, 1])
    ref = alone(wl, groups, wl.batches)
    for t, g in enumerate(groups):
        for qi, q in enumerate(g):
            o = Oracle(q, wl.data)
            for bi, b in enumerate(wl.batches):
                r = o.apply(b)
                assert ref[t][bi][qi] == (r["pos"], r["neg"]), f"tenant {t} query {qi} batch {bi}"
            o.close()


@pytest.mark.parametrize("slots,budget", [(3, 1 << 30), (2, 8 << 20), (1, 1 << 30), (4, 0x10000)])
def test_same_alone_and_in_the_mix_broadcast(wl, slots, budget):
    groups = tenant_groups(wl, [2, 3, 1])
    ref = alone(wl, groups, wl.batches)
    got, st = served(wl, groups, wl.batches, slots, budget)
    assert got == ref
    assert st.units == len(groups) * len(wl.batches)
    if slots > 1:
        assert st.peak_inflight >= 1


def test_same_alone_and_in_the_mix_interleaved(wl):
    groups = tenant_groups(wl, [1, 2, 2, 1])
    ref = alone(wl, groups, wl.batches)
    got, st = served(wl, groups, wl.batches, 3, 256 << 20, per_tenant=True)
    assert got == ref
    assert st.requests == len(groups) * len(wl.batches)


def test_depth_first_tenants_and_mixed_strategies(wl):
    # Tenants with different search strategies in one server: depth-first tenants take no
    # frontier memory, semi-BFS tenants do; counts stay those of each engine alone.
    groups = tenant_groups(wl, [3, 3])
    ref0 = alone(wl, groups[:1], wl.batches, search_strategy=0)
    ref1 = alone(wl, groups[1:], wl.batches, search_strategy=3)
    engines = [make_engine(groups[0], wl.data, search_strategy=0), make_engine(groups[1], wl.data, search_strategy=3)]
    srv = csm.Server(slots=2, memory_budget=64 << 20, min_frontier_bytes=1 << 16)
    for e in engines:
        srv.add_tenant(e)
    ids = [srv.submit(b) for b in wl.batches]
    got = []
    for rid in ids:
        info, res = srv.wait(rid)
        got.append([(r.positive, r.negative) for r in res])
    st = srv.stats()
    srv.close()
    for e in engines:
        e.close()
    assert [row[:3] for row in got] == ref0[0]
    assert [row[3:] for row in got] == ref1[0]
    assert st.units_depth_first >= len(wl.batches)


def test_engine_usable_after_server_and_errors_reported(wl):
    eng = make_engine(wl.queries[:1], wl.data)
    srv = csm.Server(slots=2)
    srv.add_tenant(eng)
    with pytest.raises(csm.CsmError):
        srv.add_tenant(eng)
    with pytest.raises(csm.CsmError):
        srv.submit(wl.batches[0], tenant=5)
    rid = srv.submit(wl.batches[0])
    info, res = srv.wait(rid)
    assert info.status == 0 and info.nresults == 1
    with pytest.raises(csm.CsmError):
        srv.wait(rid)
    srv.close()
    # After the server is gone the engine continues the stream through csm_apply_batch.
    ref = alone(wl, [wl.queries[:1]], wl.batches[:2])
    r = eng.apply(wl.batches[1])
    assert [(x.positive, x.negative) for x in r] == ref[0][1]
    eng.close()
