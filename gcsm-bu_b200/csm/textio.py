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


def _write_rows(f, tag: str, *cols) -> None:
    """Lines `tag c0 c1 ...` of integer columns (pandas' C writer for large arrays)."""
    n = len(cols[0])
    if n == 0:
        return
    if n < 100_000:
        f.write("".join(tag + " " + " ".join(str(int(c[i])) for c in cols) + "\n" for i in range(n)))
        return
    import pandas as pd
    df = pd.DataFrame({"t": np.full(n, tag, dtype=object), **{str(k): np.asarray(c, dtype=np.int64)
                                                              for k, c in enumerate(cols)}})
    df.to_csv(f, sep=" ", header=False, index=False, lineterminator="\n")


def write_graph(path: str, vlabels, src, dst, elabels, header: str = "t # 0") -> None:
    vlabels = np.asarray(vlabels)
    with open(path, "w") as f:
        f.write(header + "\n")
        _write_rows(f, "v", np.arange(len(vlabels)), vlabels)
        _write_rows(f, "e", src, dst, elabels)


def write_query(path: str, q: QueryGraph) -> None:
    write_graph(path, q.vlabels, q.src, q.dst, q.elabels)


def write_data(path: str, g: DataGraph) -> None:
    write_graph(path, g.vlabels, g.src, g.dst, g.elabels)


def write_updates(path: str, batches: Sequence[Batch]) -> None:
    with open(path, "w") as f:
        for b in batches:
            dl = b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
            if not np.any(dl):
                _write_rows(f, "e", b.src, b.dst, b.elabels)
                continue
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


# Binary forms of the data graph and the update stream (read by csmg when a file starts with
# the magic; no counterpart in the reference, whose text parsing dominates "Read Graphs from
# Files").  Little-endian:
#   data:    b"CSMBGRF1", u32 nv, u32 0, u64 ne, u32 vlabel[nv] (0xFFFFFFFF = absent),
#            u32 src[ne], u32 dst[ne], u32 elabel[ne]
#   updates: b"CSMBUPD1", u64 n, u32 src[n], u32 dst[n], u32 elabel[n], u8 is_delete[n]
# Every update record counts as one update line for the batch cut.
BIN_DATA_MAGIC = b"CSMBGRF1"
BIN_UPDATE_MAGIC = b"CSMBUPD1"


def write_binary_data(path: str, g: DataGraph) -> None:
    vl = np.ascontiguousarray(g.vlabels, dtype="<u4")
    with open(path, "wb") as f:
        f.write(BIN_DATA_MAGIC)
        f.write(np.array([len(vl), 0], dtype="<u4").tobytes())
        f.write(np.array([len(g.src)], dtype="<u8").tobytes())
        for a in (vl, g.src, g.dst, g.elabels):
            f.write(np.ascontiguousarray(a, dtype="<u4").tobytes())


def write_binary_updates(path: str, batches: Sequence[Batch]) -> None:
    src = np.concatenate([b.src for b in batches]).astype("<u4")
    dst = np.concatenate([b.dst for b in batches]).astype("<u4")
    lab = np.concatenate([b.elabels for b in batches]).astype("<u4")
    dl = np.concatenate([b.is_delete if b.is_delete is not None else np.zeros(len(b.src), dtype=np.uint8)
                         for b in batches]).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(BIN_UPDATE_MAGIC)
        f.write(np.array([len(src)], dtype="<u8").tobytes())
        for a in (src, dst, lab, dl):
            f.write(a.tobytes())


def read_binary_data(path: str):
    with open(path, "rb") as f:
        if f.read(8) != BIN_DATA_MAGIC:
            raise ValueError("not a binary data graph")
        nv, _ = np.frombuffer(f.read(8), dtype="<u4")
        (ne,) = np.frombuffer(f.read(8), dtype="<u8")
        arr = np.frombuffer(f.read(4 * (int(nv) + 3 * int(ne))), dtype="<u4")
    nv, ne = int(nv), int(ne)
    return arr[:nv], arr[nv: nv + ne], arr[nv + ne: nv + 2 * ne], arr[nv + 2 * ne:]


def read_binary_updates(path: str):
    with open(path, "rb") as f:
        if f.read(8) != BIN_UPDATE_MAGIC:
            raise ValueError("not a binary update stream")
        (n,) = np.frombuffer(f.read(8), dtype="<u8")
        n = int(n)
        arr = np.frombuffer(f.read(12 * n), dtype="<u4")
        dl = np.frombuffer(f.read(n), dtype=np.uint8)
    return arr[:n], arr[n: 2 * n], arr[2 * n:], dl
