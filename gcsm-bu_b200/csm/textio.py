"""Readers and writers of the reference's `v`/`e` text formats (graph/graph.cpp:191-563).

Query and data files: `t ...` lines are skipped, `v <id> <label>` declares a vertex, every
other line is `e <src> <dst> <label>`.  Update files hold `e <src> <dst> <label>` insertions;
`-e <src> <dst> <label>` deletions are this project's extension (the reference treats every
non-`v`, non-`t` line as an insertion and exits on vertex updates, graph.cpp:502-505).
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

from . import Batch, DataGraph, QueryGraph


def write_graph(path: str, vlabels, src, dst, elabels, header: str = "t # 0") -> None:
    vlabels = np.asarray(vlabels)
    with open(path, "w") as f:
        f.write(header + "\n")
        f.write("".join(f"v {i} {int(l)}\n" for i, l in enumerate(vlabels)))
        f.write("".join(f"e {int(a)} {int(b)} {int(l)}\n" for a, b, l in zip(src, dst, elabels)))


def write_query(path: str, q: QueryGraph) -> None:
    write_graph(path, q.vlabels, q.src, q.dst, q.elabels)


def write_data(path: str, g: DataGraph) -> None:
    write_graph(path, g.vlabels, g.src, g.dst, g.elabels)


def write_updates(path: str, batches: Sequence[Batch]) -> None:
    with open(path, "w") as f:
        for b in batches:
            dl = b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
            f.write("".join(f"{'-e' if d else 'e'} {int(x)} {int(y)} {int(l)}\n"
                            for x, y, l, d in zip(b.src, b.dst, b.elabels, dl)))


def read_graph(path: str):
    vl = {}
    src, dst, el = [], [], []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t or t[0] == "t":
                continue
            if t[0] == "v":
                vl.setdefault(int(t[1]), int(t[2]))
            else:
                src.append(int(t[1]))
                dst.append(int(t[2]))
                el.append(int(t[3]))
    n = max(vl) + 1 if vl else 0
    labels = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
    for k, v in vl.items():
        labels[k] = v
    return labels, np.array(src, dtype=np.uint32), np.array(dst, dtype=np.uint32), np.array(el, dtype=np.uint32)


def read_query(path: str) -> QueryGraph:
    return QueryGraph(*read_graph(path))


def read_updates(path: str, batch_size: int) -> List[Batch]:
    """Batch k holds update lines [k*B, (k+1)*B) (graph.cpp:507-516)."""
    rows = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t or t[0] == "t":
                continue
            rows.append((int(t[1]), int(t[2]), int(t[3]), 1 if t[0] == "-e" else 0))
    out = []
    for b0 in range(0, len(rows), batch_size):
        chunk = np.array(rows[b0:b0 + batch_size], dtype=np.uint64).reshape(-1, 4)
        dl = chunk[:, 3].astype(np.uint8)
        out.append(Batch(chunk[:, 0].astype(np.uint32), chunk[:, 1].astype(np.uint32), chunk[:, 2].astype(np.uint32),
                         dl if dl.any() else None))
    return out
