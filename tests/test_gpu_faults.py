"""GPU tests of the error paths under injected allocation failures (no GPU fault involved).

csm_config.inject_alloc_failure = N makes the engine's N-th device allocation fail as out of
memory.  Sweeping N over creation, graph load and batch-buffer growth, every call must return a
status (never abort): a failed creation or load reports CSM_ERR_OOM (a half-built engine then
refuses further calls with CSM_ERR_STATE), and a failed growth of the batch buffers leaves the
engine working at its previous capacity, so the same batch applied again counts exactly.
"""
import pytest

import csm
from helpers import small_workload

pytestmark = pytest.mark.gpu

OOM, STATE = -3, -5


def reference_counts(w, **cfg):
    with csm.Engine(**cfg) as eng:
        for q in w.queries:
            eng.load_query(q)
        eng.load_graph(w.data)
        return [[(r.positive, r.negative) for r in eng.apply(b)] for b in w.batches[:2]]


def test_injected_allocation_failures():
    w = small_workload("c2", scale=0.005, batch=700, nqueries=2)
    cfg = dict(search_strategy=2, max_batch=256)  # 700-update batches grow the batch buffers
    want = reference_counts(w, **cfg)
    seen = {"create": 0, "load": 0, "growth": 0, "none": 0}
    for n in range(1, 96):  # creation and load take ~46 allocations, growing the batch buffers ~18
        try:
            eng = csm.Engine(inject_alloc_failure=n, **cfg)
        except csm.CsmError as e:
            assert e.code == OOM
            seen["create"] += 1
            continue
        for q in w.queries:
            eng.load_query(q)
        try:
            eng.load_graph(w.data)
        except csm.CsmError as e:
            assert e.code == OOM, str(e)
            seen["load"] += 1
            with pytest.raises(csm.CsmError) as later:
                eng.apply(w.batches[0])
            assert later.value.code == STATE
            eng.close()
            continue
        try:
            got = [(r.positive, r.negative) for r in eng.apply(w.batches[0])]
            seen["none"] += 1
        except csm.CsmError as e:
            assert e.code == OOM, str(e)
            seen["growth"] += 1
            # Nothing of the batch was applied: the same batch again counts exactly.
            got = [(r.positive, r.negative) for r in eng.apply(w.batches[0])]
        assert got == want[0], n
        assert [(r.positive, r.negative) for r in eng.apply(w.batches[1])] == want[1], n
        eng.close()
    assert seen["create"] > 0 and seen["load"] > 0 and seen["growth"] > 0 and seen["none"] > 0, seen


def test_corrupt_snapshot_leaves_engine_loadable(tmp_path):
    """A rejected snapshot changes nothing: the same engine then loads a good one."""
    w = small_workload("c1", scale=0.3)
    with csm.Engine() as eng:
        eng.load_query(w.queries[0])
        eng.load_graph(w.data)
        eng.apply(w.batches[0])
        good = str(tmp_path / "good.snap")
        eng.save_snapshot(good)
        want = [(r.positive, r.negative) for r in eng.apply(w.batches[1])]
    raw = bytearray(open(good, "rb").read())
    # Layout: 48-byte header, one label byte per vertex, then the list table {offset, size}:
    # the first list's size is set beyond its capacity.
    at = 48 + len(w.data.vlabels) + 4
    raw[at:at + 4] = b"\xff\xff\xff\xff"
    bad = str(tmp_path / "bad.snap")
    open(bad, "wb").write(bytes(raw))
    with csm.Engine() as eng:
        eng.load_query(w.queries[0])
        with pytest.raises(csm.CsmError) as e:
            eng.load_snapshot(bad)
        assert e.value.code == -1
        eng.load_snapshot(good)
        assert [(r.positive, r.negative) for r in eng.apply(w.batches[1])] == want
