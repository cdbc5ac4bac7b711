"""Device recount (ccb_evaluate_labelings) against the CPU oracle's Rebuild and ObjectiveBitwise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ccb, torch, bits, edges, k, labels):
    count, n = labels.shape
    dbits = torch.from_numpy(bits.view(np.int32)).cuda()
    dlab = torch.from_numpy(labels).cuda()
    f = torch.empty(count, dtype=torch.int64, device="cuda")
    sizes = torch.empty((count, k), dtype=torch.int32, device="cuda")
    g = torch.empty((count, k, max(n, 1)), dtype=torch.int32, device="cuda")
    ccb.evaluate_labelings(dbits.data_ptr(), n, bits.shape[1], edges, k, count, dlab.data_ptr(), f.data_ptr(),
                           sizes.data_ptr(), g.data_ptr())
    torch.cuda.synchronize()
    return f.cpu().numpy(), sizes.cpu().numpy(), g.cpu().numpy()[:, :, :n]


@pytest.mark.parametrize("n,k", [(1, 1), (31, 2), (32, 3), (33, 5), (257, 7), (1000, 64), (3000, 9)])
def test_evaluate_matches_oracle(ccb, oracle, cuda_device, n, k):
    import torch
    rng = np.random.default_rng(n * 7 + k)
    bits, edges = oracle.erdos_renyi(n, 0.37, n + k)
    labels = rng.integers(0, k, (5, n)).astype(np.int32)
    f, sizes, g = _run(ccb, torch, bits, edges, k, labels)
    for i in range(labels.shape[0]):
        fo, go, so = oracle.rebuild(bits, edges, k, labels[i])
        assert f[i] == fo == oracle.objective_bitwise(bits, labels[i])
        assert np.array_equal(sizes[i], so) and np.array_equal(g[i], go)


def test_evaluate_flags_bad_labels(ccb, oracle, cuda_device):
    import torch
    bits, edges = oracle.erdos_renyi(100, 0.5, 1)
    labels = np.zeros((2, 100), np.int32)
    labels[1, 7] = 3
    f, _, _ = _run(ccb, torch, bits, edges, 3, labels)
    assert f[0] == oracle.objective_bitwise(bits, labels[0]) and f[1] == -1


def test_evaluate_recounts_a_solve(ccb, oracle, cuda_device):
    import torch
    bits, edges = oracle.erdos_renyi(2000, 0.3, 4)
    r = ccb.SolveGpu(ccb.Graph(2000, bits, edges), ccb.PbilsParams(k=6, population=32, iterations=5))
    f, _, _ = _run(ccb, torch, bits, edges, 6, r.labels.reshape(1, -1).astype(np.int32))
    assert f[0] == r.objective
