"""CPU oracle of the tags graph (test infrastructure only; the product builds it on the GPU).

Restates Graph::LoadTags of the reference (src/cc_graph.cpp:311-371) by its definition, pair by pair in numpy:
* the tags file is {"key": ["tag", ...], ...}; a vertex is an object's position in the file, tags are numbered
  by first appearance and each object's set is sorted without repeats (ReadTagSets, src/cc_graph.cpp:35-96);
* n objects are drawn by a partial Fisher-Yates shuffle on the splitmix64 stream StreamSeed(seed, 0x7A65, 0)
  with the multiply-shift RandBelow (SampleWithoutReplacement, src/cc_graph.cpp:373-381; include/cc_math.hpp);
* two objects are joined when similarity(common, |a|, |b|) >= threshold, computed in float64 with the
  reference's formulas (Similarity, src/cc_graph.cpp:107-118): jaccard inter / (a + b - common), cosine
  inter / sqrt(a * b), dice 2 inter / (a + b), overlap inter / min(a, b); 0/0 is NaN and joins nothing;
* no self loops; edges = half the sum of the degrees.
It works on the full n x n similarity matrix, so it is meant for the small fixtures of the tests.
"""
from __future__ import annotations

import json

import numpy as np

_GAMMA = 0x9E3779B97F4A7C15
_MASK = (1 << 64) - 1


def _mix(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
    return z ^ (z >> 31)


def _stream_seed(seed: int, stream: int, step: int) -> int:
    s = (seed ^ ((stream * 0xD1B54A32D192ED03) & _MASK) ^ ((step * 0xA0761D6478BD642F) & _MASK)) & _MASK
    return (s + _GAMMA) & _MASK


def read_tag_sets(path: str) -> list[list[int]]:
    with open(path) as f:
        objects = json.load(f)  # keys in file order (the fixtures have no repeated keys)
    ids: dict[str, int] = {}
    sets = []
    for tags in objects.values():
        sets.append(sorted({ids.setdefault(t, len(ids)) for t in tags}))
    return sets


def sample(total: int, n: int, seed: int) -> list[int]:
    items = list(range(total))
    if n == 0 or n >= total:
        return items
    state = _stream_seed(seed, 0x7A65, 0)
    for i in range(n):
        state = (state + _GAMMA) & _MASK
        j = i + (((_mix(state) >> 32) * (total - i)) >> 32)
        items[i], items[j] = items[j], items[i]
    return items[:n]


def load_tags(path: str, similarity: str, threshold: float, n: int, seed: int):
    """(bits [size][max(1, ceil(size/32))] uint32, edges) of the tags graph."""
    sets = read_tag_sets(path)
    objects = sample(len(sets), n, seed)
    size = len(objects)
    vocab = 1 + max((t for s in sets for t in s), default=0)
    inc = np.zeros((size, vocab), np.int32)
    for v, o in enumerate(objects):
        inc[v, sets[o]] = 1
    common = (inc @ inc.T).astype(np.float64)
    sz = inc.sum(axis=1).astype(np.float64)
    a, b = sz[:, None], sz[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        if similarity == "jaccard":
            sim = common / (a + b - common)
        elif similarity == "cosine":
            sim = common / np.sqrt(a * b)
        elif similarity == "dice":
            sim = 2.0 * common / (a + b)
        elif similarity == "overlap":
            sim = common / np.minimum(a, b)
        else:
            raise ValueError(similarity)
        adj = sim >= threshold
    np.fill_diagonal(adj, False)
    words = max(1, (size + 31) // 32)
    padded = np.zeros((size, words * 32), bool)
    padded[:, :size] = adj
    bits = np.packbits(padded, axis=1, bitorder="little").view("<u4").reshape(size, words).astype(np.uint32)
    return bits, int(adj.sum()) // 2
