"""The tags graph built on the device (ccb_graph_load_tags) against the golden graphs, which the oracle and the
reference's own Graph::LoadTags (src/cc_graph.cpp:311-371) produced and agreed on; and the loader's errors."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_G = json.load(open(os.path.join(GOLDEN, "tags_reference.json")))
SRC = os.path.join(GOLDEN, _G["file"])


@pytest.mark.parametrize("case", _G["cases"], ids=lambda c: f"{c['similarity']}_{c['threshold']}_n{c['n']}")
def test_device_tags_graph_matches_golden(ccb, cuda_device, case):
    g = ccb.DeviceGraph.load_tags(SRC, case["similarity"], case["threshold"], case["n"], case["seed"]).download()
    assert (g.n, g.edges) == (case["size"], case["edges"])
    assert hashlib.sha256(np.ascontiguousarray(g.bits, "<u4").tobytes()).hexdigest() == case["bits_sha256"]
    assert int(sum(int(x).bit_count() for x in g.bits.ravel())) == 2 * g.edges


def test_device_tags_graph_errors(ccb, cuda_device, tmp_path):
    with pytest.raises(RuntimeError, match="unknown similarity 'tanimoto'"):
        ccb.DeviceGraph.load_tags(SRC, "tanimoto", 0.5, 10, 1)
    with pytest.raises(RuntimeError, match="cannot open file"):
        ccb.DeviceGraph.load_tags(str(tmp_path / "missing.json"), "jaccard", 0.5, 10, 1)
    bad = tmp_path / "bad.json"
    bad.write_text('{"a": ["x", "y"], "b": ["x" "z"]}')
    with pytest.raises(RuntimeError, match="malformed tags json"):
        ccb.DeviceGraph.load_tags(str(bad), "jaccard", 0.5, 0, 1)
    empty = tmp_path / "empty.json"
    empty.write_text("{}")
    with pytest.raises(RuntimeError, match="no objects in"):
        ccb.DeviceGraph.load_tags(str(empty), "jaccard", 0.5, 0, 1)


def test_tags_graph_solves_like_the_oracle(ccb, oracle, cuda_device):
    """A PBILS solve on the device-built tags graph equals the oracle's on the oracle-built graph."""
    from oracle import make_params
    import tags
    bits, edges = tags.load_tags(SRC, "jaccard", 0.3, 1000, 7)
    g = ccb.DeviceGraph.load_tags(SRC, "jaccard", 0.3, 1000, 7).download()
    got = ccb.SolveGpu(g, ccb.PbilsParams(k=6, population=32, iterations=5, seed=3))
    want = oracle.pbils(bits, edges, make_params(k=6, population=32, iterations=5, seed=3))
    assert got.objective == want.objective and np.array_equal(got.labels, want.labels)
