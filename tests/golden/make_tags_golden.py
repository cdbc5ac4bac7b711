"""Golden tags graphs for the tags-graph parity tests.

    python tests/golden/make_tags_golden.py

Writes tests/golden/tags_synthetic.json, a seeded synthetic stand-in for the reference's Tags_*.json datasets
(which are not in its repository): 2500 objects with 0..7 tags from a 300-tag vocabulary drawn with Zipf-like
frequencies, repeated tags inside a set, about 40% of the objects reusing an earlier object's set (in another
order) so that tag-set classes have many members, and a few empty sets.  Then, for each case of CASES, builds
the graph with the oracle's restatement (oracle/tags.py) and, when oracle/_ref was built, with the reference's
own Graph::LoadTags (oracle/ref_shim.cpp); the two must agree.  tests/golden/tags_reference.json records the
vertex count, edge count and SHA-256 of the rows (uint32 little-endian, max(1, ceil(n/32)) words per row).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import tags as oracle_tags  # noqa: E402
from oracle import Reference  # noqa: E402

CASES = [
    dict(similarity="jaccard", threshold=0.5, n=0, seed=1),
    dict(similarity="jaccard", threshold=0.3, n=1000, seed=7),
    dict(similarity="cosine", threshold=0.4, n=2000, seed=3),
    dict(similarity="dice", threshold=0.5, n=1500, seed=11),
    dict(similarity="overlap", threshold=0.6, n=800, seed=5),
    dict(similarity="overlap", threshold=1.0, n=0, seed=1),
]


def make_synthetic(path):
    rng = np.random.default_rng(20241)
    vocab = [f"t{i}" for i in range(300)]
    weights = 1.0 / np.arange(1, 301) ** 1.1
    weights /= weights.sum()
    objects = {}
    sets = []
    for i in range(2500):
        if sets and rng.random() < 0.4:
            tags = list(sets[rng.integers(len(sets))])
            rng.shuffle(tags)
        elif rng.random() < 0.03:
            tags = []
        else:
            count = int(rng.integers(1, 8))
            tags = [vocab[j] for j in rng.choice(300, size=count, p=weights)]  # may repeat a tag
        sets.append(tags)
        objects[f"obj{i}"] = tags
    with open(path, "w") as f:
        json.dump(objects, f, separators=(",", ":"))
    return len(objects)


def main():
    src = os.path.join(HERE, "tags_synthetic.json")
    total = make_synthetic(src)
    ref = Reference() if Reference.available() else None
    out = dict(file="tags_synthetic.json", objects=total, checked_against_reference=ref is not None, cases=[])
    for c in CASES:
        bits, edges = oracle_tags.load_tags(src, c["similarity"], c["threshold"], c["n"], c["seed"])
        if ref is not None:
            rbits, redges = ref.load_tags(src, c["similarity"], c["threshold"], c["n"], c["seed"], total)
            assert redges == edges and np.array_equal(rbits, bits), c
        sha = hashlib.sha256(np.ascontiguousarray(bits, "<u4").tobytes()).hexdigest()
        out["cases"].append(dict(c, size=int(bits.shape[0]), edges=edges, bits_sha256=sha))
        print(out["cases"][-1], flush=True)
    with open(os.path.join(HERE, "tags_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
