"""The csmg drop-in: reference flags and text formats in, the reference's result lines out."""
import os
import re
import subprocess

import numpy as np
import pytest

import csm
from csm import Batch, textio
from oracle import Oracle
from helpers import small_workload

pytestmark = pytest.mark.gpu


def run_csmg(tmp_path, w, extra=(), batches=None, query=None):
    query = w.queries[0] if query is None else query
    batches = w.batches if batches is None else batches
    qf, df, uf = (str(tmp_path / x) for x in ("q.graph", "d.graph", "u.graph"))
    textio.write_query(qf, query)
    textio.write_data(df, w.data)
    textio.write_updates(uf, batches)
    bs = max(len(b.src) for b in batches)
    p = subprocess.run([csm.CSMG_PATH, "--query", qf, "--data", df, "--update", uf, "--batch_size", str(bs), *extra],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    return p.stdout


def totals(w, batches=None, query=None):
    o = Oracle(w.queries[0] if query is None else query, w.data)
    pos = neg = 0
    for b in (w.batches if batches is None else batches):
        r = o.apply(b)
        pos += r["pos"]
        neg += r["neg"]
    return pos, neg


@pytest.mark.parametrize("extra", [(), ("--algorithm", "1"), ("--algorithm", "2"),
                                   ("--search_strategy", "0", "--cartesian_product", "False"),
                                   ("--matching_order", "3", "--local_index", "false")])
def test_csmg_insert_only(tmp_path, extra):
    w = small_workload("c1")
    out = run_csmg(tmp_path, w, extra)
    pos, _ = totals(w)
    assert re.search(r"^Num Positive Matches: (\d+)$", out, re.M).group(1) == str(pos)
    assert re.search(r"^Incremental Matching, time \(ms\): \d+\(host\), \d+\(kernel\)$", out, re.M)
    assert len(re.findall(r"^Batch #\d+ --------$", out, re.M)) == len(w.batches)


def test_csmg_with_deletions(tmp_path):
    w = small_workload("c2", scale=0.002, batch=300, nqueries=2)
    out = run_csmg(tmp_path, w)
    pos, neg = totals(w)
    assert re.search(r"^Num Positive Matches: (\d+)$", out, re.M).group(1) == str(pos)
    assert re.search(r"^Num Negative Matches: (\d+)$", out, re.M).group(1) == str(neg)
    assert neg > 0


def batch_lines(out):
    return re.findall(r"^Batch #\d+: pos=(\d+) neg=(\d+) ins=(\d+) del=(\d+)", out, re.M)


def test_csmg_binary_inputs_match_text(tmp_path):
    w = small_workload("c2", scale=0.002, batch=300, nqueries=1)
    text_out = run_csmg(tmp_path, w)
    qf, df, uf = (str(tmp_path / x) for x in ("q.graph", "d.bin", "u.bin"))
    textio.write_query(qf, w.queries[0])
    textio.write_binary_data(df, w.data)
    textio.write_binary_updates(uf, w.batches)
    bs = max(len(b.src) for b in w.batches)
    p = subprocess.run([csm.CSMG_PATH, "--query", qf, "--data", df, "--update", uf, "--batch_size", str(bs)],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-3000:]
    assert batch_lines(p.stdout) == batch_lines(text_out) and len(batch_lines(text_out)) == len(w.batches)


def test_csmg_snapshot_resume(tmp_path):
    # First half of the stream, snapshot, then the second half from the snapshot: the same
    # per-batch lines as one uninterrupted run.
    w = small_workload("c2", scale=0.002, batch=300, nqueries=1)
    full = batch_lines(run_csmg(tmp_path, w))
    half = len(w.batches) // 2
    snap = str(tmp_path / "g.snap")
    first = batch_lines(run_csmg(tmp_path, w, ("--snapshot_out", snap), batches=w.batches[:half]))
    second = batch_lines(run_csmg(tmp_path, w, ("--snapshot_in", snap), batches=w.batches[half:]))
    assert first + second == full
