"""The oracle pinned against the reference itself: tests/golden/reference_counts.json holds the
"Num Positive Matches" totals of the reference GCSM-BU built for sm_100a (made by
tests/golden/make_golden.py on a B200) for seeded insert-only streams."""
import json
import os

import pytest

from oracle import Oracle
from golden_cases import CASES, build_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_counts.json")


def load():
    with open(GOLDEN) as f:
        return {e["id"]: e for e in json.load(f)}


def test_fixture_covers_every_case():
    g = load()
    assert sorted(g) == sorted(c["id"] for c in CASES)


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_oracle_matches_reference(case):
    entry = load()[case["id"]]
    query, data, batches, _ = build_case(case)
    o = Oracle(query, data)
    per_batch = [o.apply(b)["pos"] for b in batches]
    assert per_batch == entry["oracle_per_batch"]
    for alg in case["algorithms"]:
        assert entry[f"reference_alg{alg}_rc"] == 0
        assert entry[f"reference_alg{alg}"] == sum(per_batch), f"algorithm {alg}"
