"""Times the reference GCSM-BU build (oracle/_ref/csmg_ref, compiled for sm_100a from the
reference sources) against this project's csmg on identical insert-only input files.

Both tools print the reference's result lines, so the comparison reads the same
"Incremental Matching, time (ms): H(host), K(kernel)" and "Num Positive Matches" lines from
each.  Needs a B200.  Usage: python oracle/time_reference.py [out.json [name:config:scale:batch:q,q:timeout ...]]
"""
import json
import os
import re
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gcsm-bu_b200"))

from csm import CSMG_PATH, gen, textio  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "csmg_ref")

# (name, config, scale, batch, query indices, per-run timeout in seconds)
RUNS = [
    ("c1", "c1", 1.0, 1024, [0], 300),
    ("c2@0.05", "c2", 0.05, 3277, list(range(10)), 120),
    ("c2@0.2", "c2", 0.2, 13107, list(range(5)), 180),
]


def run(cmd, timeout):
    t0 = time.time()
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"timeout": timeout}
    wall = time.time() - t0
    m = re.search(r"^Incremental Matching, time \(ms\): (\d+)\(host\), (\d+)\(kernel\)", p.stdout, re.M)
    c = re.search(r"^Num Positive Matches: (\d+)", p.stdout, re.M)
    return {"rc": p.returncode, "host_ms": int(m.group(1)) if m else None, "kernel_ms": int(m.group(2)) if m else None,
            "positive": int(c.group(1)) if c else None, "wall_s": round(wall, 2)}


def parse_runs(specs):
    """name:config:scale:batch:q,q,...:timeout"""
    runs = []
    for sp in specs:
        name, cname, scale, batch, qs, tmo = sp.split(":")
        runs.append((name, cname, float(scale), int(batch), [int(x) for x in qs.split(",")], int(tmo)))
    return runs


def main():
    out_path = sys.argv[1] if len(sys.argv) > 1 else "reference_timing.json"
    runs = parse_runs(sys.argv[2:]) if len(sys.argv) > 2 else RUNS
    results = []
    with tempfile.TemporaryDirectory() as td:
        for name, cname, scale, batch, qids, tmo in runs:
            cfg = gen.scaled(cname, scale) if scale != 1.0 else dict(gen.CONFIGS[cname])
            cfg["n_del"] = 0
            cfg["batch"] = batch
            w = gen.make_workload(cname, cfg)
            df, uf = os.path.join(td, "d.graph"), os.path.join(td, "u.graph")
            textio.write_data(df, w.data)
            textio.write_updates(uf, w.batches)
            for qi in qids:
                qf = os.path.join(td, f"q{qi}.graph")
                textio.write_query(qf, w.queries[qi])
                args = ["--query", qf, "--data", df, "--update", uf, "--batch_size", str(batch), "--algorithm", "1"]
                ref = run([REF] + args, tmo)
                ours = run([CSMG_PATH] + args, tmo)
                row = {"workload": name, "query": qi, "query_edges": int(len(w.queries[qi].src)),
                       "batches": len(w.batches), "reference": ref, "ours": ours}
                results.append(row)
                print(json.dumps(row), flush=True)
    with open(out_path, "w") as f:
        json.dump(results, f, indent=1)


if __name__ == "__main__":
    main()
