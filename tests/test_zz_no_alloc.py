"""The allocation-free recount (ccb_evaluate_labelings_noalloc) against the allocating one.

Callers that cannot allocate device memory when they call in (device memory already reserved by their
own pool allocator, or a loop that must not pay cudaMalloc/cudaFree) use the no-alloc entry point, whose
scratch is a fixed device array shared by all calls.  Two calls in a row with different inputs must each
give exactly the allocating entry point's output (integer results: the tolerance is zero), so nothing
left in the shared scratch by one call leaks into the next.  This file is collected last so that a run
that stops at the first failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_inputs(torch, oracle, n, k, count, graph_seed, label_seed):
    bits, edges = oracle.erdos_renyi(n, 0.41, graph_seed)
    labels = np.random.default_rng(label_seed).integers(0, k, (count, n)).astype(np.int32)
    return bits, edges, torch.from_numpy(bits.view(np.int32)).cuda(), torch.from_numpy(labels).cuda()


def _outputs(torch, count, k, n):
    return (torch.full((count,), -7, dtype=torch.int64, device="cuda"),
            torch.full((count, k), -7, dtype=torch.int32, device="cuda"),
            torch.full((count, k, n), -7, dtype=torch.int32, device="cuda"))


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(ccb, oracle, cuda_device):
    import torch
    # a count = 0 call is the per-device set-up (symbol lookup, module load) and touches no pointer
    ccb.evaluate_labelings_noalloc(0, 0, 0, 0, 2, 0, 0, 0)
    for n, k, count, gseed, lseed in [(1500, 9, 6, 3, 4), (700, 4, 11, 5, 6)]:
        bits, edges, dbits, dlab = _device_inputs(torch, oracle, n, k, count, gseed, lseed)
        f0, s0, g0 = _outputs(torch, count, k, n)
        f1, s1, g1 = _outputs(torch, count, k, n)
        ccb.evaluate_labelings_noalloc(dbits.data_ptr(), n, bits.shape[1], edges, k, count, dlab.data_ptr(),
                                       f1.data_ptr(), s1.data_ptr(), g1.data_ptr())
        ccb.evaluate_labelings(dbits.data_ptr(), n, bits.shape[1], edges, k, count, dlab.data_ptr(), f0.data_ptr(),
                               s0.data_ptr(), g0.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(f0, f1) and torch.equal(s0, s1) and torch.equal(g0, g1)
        assert int(f1[0]) == oracle.objective_bitwise(bits, dlab[0].cpu().numpy())


def test_noalloc_rejects_batches_beyond_its_scratch(ccb, oracle, cuda_device):
    import torch
    n, k, count = 32768, 64, 17  # 17 * 64 * 1024 words > 1048576
    f = torch.empty(count, dtype=torch.int64, device="cuda")
    with pytest.raises(RuntimeError) as e:
        ccb.evaluate_labelings_noalloc(f.data_ptr(), n, n // 32, 0, k, count, f.data_ptr(), f.data_ptr())
    assert "exceeds the 1048576 mask words" in str(e.value)


def test_noalloc_full_scratch_without_optional_outputs(ccb, oracle, cuda_device):
    """A batch that fills the scratch exactly (32 * 64 * 512 = 1048576 mask words, the last word included),
    with sizes_out and g_out NULL, twice in a row: f equals the allocating entry point's."""
    import torch
    n, k, count = 16384, 64, 32
    assert count * k * ((n + 31) // 32) == 1 << 20
    for gseed, lseed in [(11, 12), (13, 14)]:
        bits, edges = oracle.erdos_renyi(n, 0.03, gseed)
        labels = np.random.default_rng(lseed).integers(0, k, (count, n)).astype(np.int32)
        labels[-1, -32:] = k - 1  # the last labeling's last word: the array's final mask word is nonzero
        dbits = torch.from_numpy(bits.view(np.int32)).cuda()
        dlab = torch.from_numpy(labels).cuda()
        f0 = torch.full((count,), -7, dtype=torch.int64, device="cuda")
        f1 = torch.full((count,), -7, dtype=torch.int64, device="cuda")
        ccb.evaluate_labelings_noalloc(dbits.data_ptr(), n, bits.shape[1], edges, k, count, dlab.data_ptr(),
                                       f1.data_ptr())
        ccb.evaluate_labelings(dbits.data_ptr(), n, bits.shape[1], edges, k, count, dlab.data_ptr(), f0.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(f0, f1)
        assert int(f1[-1]) == oracle.objective_bitwise(bits, labels[-1])
