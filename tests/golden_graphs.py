"""Small graph builders shared by the tests."""
import numpy as np


def graph_from_mask(n: int, mask: int) -> np.ndarray:
    """Graph on n vertices whose pairs (v < u, v ascending then u ascending) are edges where `mask` has a
    bit, as in the exhaustive loop of the reference's GPU test (cuda/cc_verify_gpu.cu:88-100)."""
    words = max(1, (n + 31) // 32)
    bits = np.zeros((n, words), np.uint32)
    bit = 0
    for v in range(n):
        for u in range(v + 1, n):
            if (mask >> bit) & 1:
                bits[v, u // 32] |= np.uint32(1 << (u % 32))
                bits[u, v // 32] |= np.uint32(1 << (v % 32))
            bit += 1
    return bits
