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
