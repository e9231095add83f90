"""csm_apply_batch_device_static, the entry point for callers that cannot allocate device memory
while they apply updates (processes that reserve their whole memory budget up front, or hosts
that own all device memory).  Its results must equal csm_apply_batch_device's, batch after
batch, and it must refuse work that does not fit its fixed scratch instead of allocating.

Collected last on purpose: a run that stops at its first failure has run everything else."""
import numpy as np
import pytest

import csm
from helpers import small_workload

pytestmark = pytest.mark.gpu


def device_batch(b, torch):
    dl = b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda()
            for a in (b.src.astype(np.int32), b.dst.astype(np.int32), b.elabels.astype(np.int32), dl)]


def loaded_engine(w, **cfg):
    eng = csm.Engine(**cfg)
    for q in w.queries:
        eng.load_query(q)
    eng.load_graph(w.data)
    return eng


def test_static_entry_matches_allocating_entry_on_consecutive_batches():
    import torch
    w = small_workload("c2", scale=0.005, batch=700, nqueries=3)
    ref = loaded_engine(w, max_batch=4096)
    sta = loaded_engine(w, max_batch=4096)
    stream = torch.cuda.current_stream().cuda_stream
    for b in w.batches[:2]:
        s, d, l, dl = device_batch(b, torch)
        ptrs = (len(b.src), s.data_ptr(), d.data_ptr(), l.data_ptr(), dl.data_ptr())
        ra = ref.apply_device(*ptrs, stream=stream)
        rb = sta.apply_device_static(*ptrs, stream=stream)
        for qi in range(len(w.queries)):
            got = (rb[qi].positive, rb[qi].negative, rb[qi].inserted, rb[qi].deleted)
            want = (ra[qi].positive, ra[qi].negative, ra[qi].inserted, ra[qi].deleted)
            assert got == want, f"query {qi}"
            assert sta.edge_counts(qi) == ref.edge_counts(qi)
    assert sum(r.positive for r in ra) > 0
    ref.close()
    sta.close()


def test_static_entry_refuses_batches_beyond_its_capacity():
    import torch
    w = small_workload("c2", scale=0.005, batch=2000, nqueries=1)
    eng = loaded_engine(w, max_batch=1024)
    b = w.batches[0]
    s, d, l, dl = device_batch(b, torch)
    with pytest.raises(csm.CsmError) as ei:
        eng.apply_device_static(len(b.src), s.data_ptr(), d.data_ptr(), l.data_ptr(), dl.data_ptr())
    assert ei.value.code == -6 and "preallocated" in str(ei.value)
    eng.close()


def test_static_entry_depth_first_with_donation_matches():
    """A depth-first strategy donates work through the library's fixed ring."""
    import torch
    w = small_workload("c2", scale=0.01, batch=1500, nqueries=4)
    ref = loaded_engine(w, max_batch=4096, search_strategy=0, steal_chunk=8)
    sta = loaded_engine(w, max_batch=4096, search_strategy=0, steal_chunk=8)
    for b in w.batches[:2]:
        s, d, l, dl = device_batch(b, torch)
        ptrs = (len(b.src), s.data_ptr(), d.data_ptr(), l.data_ptr(), dl.data_ptr())
        ra, rb = ref.apply_device(*ptrs), sta.apply_device_static(*ptrs)
        assert [(r.positive, r.negative) for r in ra] == [(r.positive, r.negative) for r in rb]
    assert sta.stats().donations > 0
    ref.close()
    sta.close()


def test_static_entry_refuses_more_query_edges_than_its_scratch_holds():
    """114 standing 9-cliques have 4104 query edges, more than the 4096 the scratch holds."""
    import torch
    from helpers import clique
    w = small_workload("c1", scale=0.3)
    eng = csm.Engine(max_batch=4096)
    for _ in range(114):
        eng.load_query(clique(9))
    eng.load_graph(w.data)
    b = w.batches[0]
    s, d, l, dl = device_batch(b, torch)
    with pytest.raises(csm.CsmError) as ei:
        eng.apply_device_static(len(b.src), s.data_ptr(), d.data_ptr(), l.data_ptr(), dl.data_ptr())
    assert ei.value.code == -6 and "4096" in str(ei.value)
    eng.close()


def test_static_entry_refuses_a_batch_the_pool_may_not_hold():
    """The call never compacts or grows the adjacency pool: with too little free room it refuses
    before changing anything, and the allocating entry point then applies the same batch."""
    import torch
    w = small_workload("c2", scale=0.005, batch=700, nqueries=2)
    probe = loaded_engine(w, max_batch=4096)
    used = probe.stats().pool_used
    probe.close()
    # Room for the graph but less than the 64 entries per update plus 2^20 the call asks for.
    eng = loaded_engine(w, max_batch=4096, pool_entries=used + (1 << 20))
    ref = loaded_engine(w, max_batch=4096)
    cap = eng.stats().pool_capacity
    b = w.batches[0]
    s, d, l, dl = device_batch(b, torch)
    ptrs = (len(b.src), s.data_ptr(), d.data_ptr(), l.data_ptr(), dl.data_ptr())
    with pytest.raises(csm.CsmError) as ei:
        eng.apply_device_static(*ptrs)
    assert ei.value.code == -6 and "pool" in str(ei.value)
    assert eng.stats().pool_capacity == cap
    got = [(r.positive, r.negative) for r in eng.apply_device(*ptrs)]
    assert got == [(r.positive, r.negative) for r in ref.apply_device(*ptrs)]
    eng.close()
    ref.close()
