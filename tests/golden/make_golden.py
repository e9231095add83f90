"""Generates tests/golden/reference_counts.json: per-case totals of the reference GCSM-BU itself.

Runs the reference binary built from the reference sources for sm_100a (oracle/_ref/csmg_ref,
built by `make -C oracle ref`) on small seeded insert-only streams — the only form the reference
reads (graph/graph.cpp:482-563) — and records its "Num Positive Matches" total
(technique_permutation.h:224) next to the CPU oracle's total for the same input.  Needs a GPU;
run it once on a B200 box:  python tests/golden/make_golden.py [out.json]
"""
import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "gcsm-bu_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

from csm import textio  # noqa: E402
from oracle import Oracle  # noqa: E402
from golden_cases import CASES, build_case  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "csmg_ref")


def run_reference(qf, df, uf, batch_size, algorithm):
    cmd = [REF, "--query", qf, "--data", df, "--update", uf, "--batch_size", str(batch_size),
           "--algorithm", str(algorithm)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    m = re.search(r"Num Positive Matches: (\d+)", p.stdout)
    return (int(m.group(1)) if m else None), p.returncode, p.stdout[-2000:] + p.stderr[-2000:]


def main():
    out_path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "reference_counts.json")
    results = []
    with tempfile.TemporaryDirectory() as td:
        for case in CASES:
            query, data, batches, bs = build_case(case)
            qf, df, uf = (os.path.join(td, f"{case['id']}.{x}") for x in ("q", "d", "u"))
            textio.write_query(qf, query)
            textio.write_data(df, data)
            textio.write_updates(uf, batches)
            o = Oracle(query, data)
            per_batch = [o.apply(b)["pos"] for b in batches]
            entry = dict(case)
            entry["oracle_total"] = int(sum(per_batch))
            entry["oracle_per_batch"] = [int(x) for x in per_batch]
            for alg in case.get("algorithms", [1]):
                cnt, rc, tail = run_reference(qf, df, uf, bs, alg)
                entry[f"reference_alg{alg}"] = cnt
                entry[f"reference_alg{alg}_rc"] = rc
                if cnt is None or rc != 0:
                    entry[f"reference_alg{alg}_log"] = tail
            results.append(entry)
            print(entry["id"], entry["oracle_total"], {k: v for k, v in entry.items() if k.startswith("reference_alg")
                                                      and not k.endswith("_log")}, flush=True)
    with open(out_path, "w") as f:
        json.dump(results, f, indent=1)


if __name__ == "__main__":
    main()
