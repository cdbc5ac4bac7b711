"""The tags-graph oracle (oracle/tags.py) against the golden graphs and the reference's own Graph::LoadTags."""
import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_G = json.load(open(os.path.join(GOLDEN, "tags_reference.json")))
SRC = os.path.join(GOLDEN, _G["file"])


@pytest.mark.parametrize("case", _G["cases"], ids=lambda c: f"{c['similarity']}_{c['threshold']}_n{c['n']}")
def test_tags_oracle_matches_golden(case):
    import tags
    bits, edges = tags.load_tags(SRC, case["similarity"], case["threshold"], case["n"], case["seed"])
    assert (bits.shape[0], edges) == (case["size"], case["edges"])
    assert hashlib.sha256(np.ascontiguousarray(bits, "<u4").tobytes()).hexdigest() == case["bits_sha256"]


def test_tags_oracle_matches_reference_loader(reference):
    import tags
    for sim, thr, n, seed in [("jaccard", 0.25, 300, 2), ("cosine", 0.7, 0, 4), ("overlap", 0.5, 1234, 9)]:
        want = reference.load_tags(SRC, sim, thr, n, seed, _G["objects"])
        got = tags.load_tags(SRC, sim, thr, n, seed)
        assert got[1] == want[1] and np.array_equal(got[0], want[0]), (sim, thr, n)
