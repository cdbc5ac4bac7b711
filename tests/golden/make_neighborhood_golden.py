"""Golden Neighborhood results at the Neighborhood configuration's size, for the GPU parity test.

    python tests/golden/make_neighborhood_golden.py

The instance: the planted two-community graph of n = 4096 vertices, split 2048/2048 by a seeded random
permutation, edge probability 0.6 inside a community and 0.1 across (oracle.planted, graph seed 1).  Both
Neighborhood algorithms (without and with the local search after every start partition) are solved by the
oracle's restatement of the brute force of cuda/cc_verify_gpu.cu:21-35 and, when oracle/_ref was built, by
the reference's own CPU code (oracle/ref_shim.cpp: the same loop over the reference's State::Rebuild and
LocalSearch); the two must agree before anything is written.  Recorded per algorithm: objective, accepted
moves, clusters used, local searches, the labels' SHA-256 (int32, little-endian) and the tie-break vertex
(the smallest start vertex whose partition, before any local search, is the chosen one; only for the plain
algorithm, where the partition identifies it).  Output: tests/golden/neighborhood_reference.json.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

from oracle import Oracle, Reference  # noqa: E402

INSTANCE = dict(n=4096, parts=2, shuffle_split=True, p_in=0.6, p_out=0.1, flip=0.0, graph_seed=1)


def _sha(labels):
    return hashlib.sha256(np.asarray(labels, dtype="<i4").tobytes()).hexdigest()


def _tie_break_vertex(bits, labels):
    """Smallest v whose start partition {v} + N(v) (label 0) against the rest equals `labels`."""
    n = bits.shape[0]
    zero = np.asarray(labels) == 0
    for v in np.flatnonzero(zero):
        row = np.unpackbits(bits[v].view(np.uint8), bitorder="little")[:n].astype(bool)
        row[v] = True
        if np.array_equal(row, zero):
            return int(v)
    return -1


def main():
    orc = Oracle()
    i = INSTANCE
    bits, edges, _ = orc.planted(i["n"], i["parts"], i["shuffle_split"], i["p_in"], i["p_out"], i["flip"],
                                 i["graph_seed"])
    ref = Reference() if Reference.available() else None
    out = dict(INSTANCE, edges=edges, checked_against_reference=ref is not None)
    for key, ls in (("plain", False), ("local_search", True)):
        got = orc.neighborhood(bits, edges, ls)
        if ref is not None:
            want = ref.neighborhood(bits, ls)
            assert (got.objective, got.accepted_moves, got.clusters_used, got.local_searches) == \
                (want.objective, want.accepted_moves, want.clusters_used, want.local_searches), key
            assert np.array_equal(got.labels, want.labels), key
        out[key] = dict(objective=int(got.objective), accepted_moves=int(got.accepted_moves),
                        clusters_used=int(got.clusters_used), local_searches=int(got.local_searches),
                        labels_sha256=_sha(got.labels))
        if not ls:
            out[key]["tie_break_vertex"] = _tie_break_vertex(bits, got.labels)
        print(key, out[key], flush=True)
    with open(os.path.join(HERE, "neighborhood_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
