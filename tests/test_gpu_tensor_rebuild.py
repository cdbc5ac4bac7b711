"""The tensor-core rebuild (int8 tcgen05 contraction fed by TMA) against the popcount rebuild.

G = A*Z counts are integers, so the two paths must agree exactly:
* the recount entry points: ccb_evaluate_labelings_tensor against ccb_evaluate_labelings (G, sizes, f) on ragged
  shapes (n not a multiple of 128, column blocks not a multiple of 16), a large population * k (many column
  blocks), and the wide configuration's size (n = 65536, p = 0.02, 128 labelings of k = 2 and k = 3);
* whole solves: a solver switched to CCB_REBUILD_TENSOR follows the popcount solver's trajectory and the
  oracle's (generic wide kernel at small n) and, at n = 65536, the reference binary's golden runs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import make_params

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _recount_both(ccb, torch, dg, n, k, count, seed):
    g = dg.download()
    words = g.bits.shape[1]
    pitch = (words + 3) // 4 * 4  # 16-byte rows, as the tensor path's TMA reads them
    padded = np.zeros((n, pitch), np.uint32)
    padded[:, :words] = g.bits
    bits = torch.from_numpy(padded.view(np.int32)).cuda()
    labels = torch.from_numpy(np.random.default_rng(seed).integers(0, k, (count, n)).astype(np.int32)).cuda()
    out = []
    for fn in (ccb.evaluate_labelings, ccb.evaluate_labelings_tensor):
        f = torch.full((count,), -7, dtype=torch.int64, device="cuda")
        sizes = torch.full((count, k), -7, dtype=torch.int32, device="cuda")
        gg = torch.full((count, k, n), -7, dtype=torch.int32, device="cuda")
        fn(bits.data_ptr(), n, pitch, g.edges, k, count, labels.data_ptr(), f.data_ptr(), sizes.data_ptr(),
           gg.data_ptr())
        torch.cuda.synchronize()
        out.append((f, sizes, gg))
    return g, labels, out


@pytest.mark.parametrize("n,k,count,density", [
    (128, 2, 1, 0.5),        # one tile, one 16-column block
    (1000, 5, 7, 0.3),       # ragged rows and K, 35 columns in a 48-column block
    (4100, 3, 100, 0.1),     # 300 columns: two blocks of 160
    (2000, 64, 64, 0.4),     # 4096 columns: 16 blocks of 256
    (33000, 9, 20, 0.01),    # 180 columns, 258 row tiles
])
def test_tensor_recount_equals_popcount(ccb, oracle, cuda_device, n, k, count, density):
    import torch
    dg = ccb.DeviceGraph.erdos_renyi(n, density, n + k)
    g, labels, ((f0, s0, g0), (f1, s1, g1)) = _recount_both(ccb, torch, dg, n, k, count, 7)
    assert torch.equal(g0, g1)
    assert torch.equal(s0, s1)
    assert torch.equal(f0, f1)
    if n <= 4100:
        assert int(f1[0]) == oracle.objective_bitwise(g.bits, labels[0].cpu().numpy())


@pytest.mark.parametrize("k", [2, 3])
def test_tensor_recount_at_the_wide_size(ccb, cuda_device, k):
    """n = 65536, p = 0.02 (the wide configuration's graph), 128 labelings: the population's whole rebuild."""
    import torch
    dg = ccb.DeviceGraph.erdos_renyi(65536, 0.02, 1)
    _, _, ((f0, s0, g0), (f1, s1, g1)) = _recount_both(ccb, torch, dg, 65536, k, 128, 3)
    assert torch.equal(f0, f1) and torch.equal(s0, s1)
    assert torch.equal(g0, g1)


@pytest.mark.parametrize("n,k,pop,density", [(300, 2, 16, 0.4), (1000, 3, 24, 0.3), (700, 9, 8, 0.5)])
def test_tensor_rebuild_solver_matches_oracle(ccb, oracle, cuda_device, n, k, pop, density):
    """The generic wide kernel (ls_kernel wide: int32 G, tiled rebuild) with either rebuild follows the oracle."""
    bits, edges = oracle.erdos_renyi(n, density, 40 + n)
    dg = ccb.DeviceGraph(ccb.Graph(n, bits, edges))
    p = ccb.PbilsParams(k=k, population=pop, iterations=6, early_stop=6, gww=0.25, seed=5, ls_kernel=3)
    want = oracle.pbils(bits, edges, make_params(k=k, population=pop, iterations=6, early_stop=6, gww=0.25, seed=5))
    for kind in ("popcount", "tensor"):
        s = ccb.Solver(dg, p)
        s.set_rebuild(kind)
        assert ("tensor cores" in s.describe()) == (kind == "tensor")
        got = s.pbils(p)
        s.close()
        assert (got.objective, got.iterations_done, got.accepted_moves) == \
            (want.objective, want.iterations_done, want.accepted_moves), kind
        assert np.array_equal(got.labels, want.labels), kind


def test_tensor_rebuild_rejected_off_the_wide_path(ccb, oracle, cuda_device):
    bits, edges = oracle.erdos_renyi(500, 0.3, 1)
    s = ccb.Solver(ccb.DeviceGraph(ccb.Graph(500, bits, edges)), ccb.PbilsParams(k=4, population=8))
    with pytest.raises(RuntimeError) as e:
        s.set_rebuild("tensor")
    assert "wide path" in str(e.value)
    s.close()


_WIDE = [r for r in json.load(open(os.path.join(GOLDEN, "wide_reference.json"))) if r["n"] == 65536]


@pytest.mark.parametrize("run", _WIDE, ids=lambda r: f"k{r['k']}_p{r['density']}")
def test_tensor_rebuild_matches_the_reference_binary_at_65536(ccb, cuda_device, run):
    dg = ccb.DeviceGraph.erdos_renyi(run["n"], run["density"], run["graph_seed"])
    p = ccb.PbilsParams(k=run["k"], population=run["population"], iterations=run["iterations"], seed=run["seed"])
    s = ccb.Solver(dg, p)
    s.set_rebuild("tensor")
    got = s.pbils(p)
    s.close()
    assert (got.objective, got.iterations_done, got.clusters_used) == \
        (run["objective"], run["iterations_done"], run["clusters_used"])
    assert hashlib.sha256(np.asarray(got.labels, dtype="<i4").tobytes()).hexdigest() == run["labels_sha256"]
