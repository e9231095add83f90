"""Runs one synthetic workload through the engine and prints one line per batch.

    python -m csm.run --config c2 --scale 0.5 --batch 32768 --insert-only --query 3 --batches 2 \
        [--set key=value ...]

Queries are selected with --query (repeatable; all by default) and registered in one engine;
`--set` overrides csm_config fields (e.g. search_strategy=0, occupancy=5, cuda_graphs=1).
Used for profiling single workloads with ncu.
"""
from __future__ import annotations

import argparse
import sys

from . import Engine, gen


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c2")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--batch", type=int, default=None)
    ap.add_argument("--insert-only", action="store_true")
    ap.add_argument("--query", type=int, action="append", default=None)
    ap.add_argument("--batches", type=int, default=None)
    ap.add_argument("--set", action="append", default=[], help="csm_config field=value")
    a = ap.parse_args(argv)
    cfg = gen.scaled(a.config, a.scale) if a.scale != 1.0 else dict(gen.CONFIGS[a.config])
    if a.batch:
        cfg["batch"] = a.batch
    if a.insert_only:
        cfg["n_del"] = 0
    w = gen.make_workload(a.config, cfg)
    overrides = {}
    for kv in a.set:
        k, v = kv.split("=", 1)
        overrides[k] = int(v)
    eng = Engine(**overrides)
    qids = a.query if a.query else list(range(len(w.queries)))
    for qi in qids:
        eng.load_query(w.queries[qi])
    eng.load_graph(w.data)
    batches = w.batches if a.batches is None else w.batches[: a.batches]
    for bi, b in enumerate(batches):
        res = eng.apply(b)
        pos = sum(r.positive for r in res)
        neg = sum(r.negative for r in res)
        print(f"batch {bi}: updates {len(b.src)} positive {pos} negative {neg} "
              f"latency_ms {res[0].latency_ns / 1e6:.3f} enum_ms {res[0].enum_ns / 1e6:.3f}", flush=True)
    st = eng.stats()
    print(f"stats: scans {st.enum_scan_entries} probes {st.enum_probes} tail_lists {st.enum_tail_lists} "
          f"donations {st.donations} kernel_launches {st.kernel_launches}", flush=True)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
