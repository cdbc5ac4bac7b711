"""Measured copy bandwidths of this GPU: L2-resident and HBM, the denominators of the roofline fractions.

    python -m cuda_graph_clustering_b200.peaks > profiles/peaks_l2_hbm.txt

A device-to-device copy (read + write, both counted) of a buffer pair, timed with CUDA events over many
repetitions after a warm-up: pairs of 2 x 16 / 32 / 48 MiB stay in the 126 MB L2 between repetitions (their
copies captured in one CUDA graph; the L2 figure is their best), a pair of 2 x 2 GiB streams from HBM.  A dense int8 GEMM (cuBLASLt) gives the int8
tensor-core peak of the tensor rebuild's roofline.  The driver-written HBM figure (a STREAM-style
copy) is the HBM peak of record; this one is printed beside it as a cross-check.  One JSON object per line,
then a summary line that bench.py reads ("l2_copy_gbs: ...").
"""
from __future__ import annotations

import json


def copy_gbs(torch, nbytes: int, reps: int, graph: bool = False) -> float:
    """Read + write bandwidth of `reps` back-to-back copies; with `graph` they are captured in one CUDA graph so
    that host launch gaps do not count (the L2-resident copies last only microseconds each)."""
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda").fill_(1)
    dst = torch.empty_like(src)
    for _ in range(5):
        dst.copy_(src)
    run = None
    if graph:
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            with torch.cuda.graph(g):
                for _ in range(reps):
                    dst.copy_(src)
        torch.cuda.current_stream().wait_stream(side)
        g.replay()
        run = g.replay
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    if run is not None:
        run()
    else:
        for _ in range(reps):
            dst.copy_(src)
    stop.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    return 2.0 * nbytes * reps / (ms * 1e-3) / 1e9


def int8_tops(torch, size: int, reps: int) -> float:
    """Dense int8 x int8 -> int32 GEMM (cuBLASLt through torch._int_mm), size^3, tera-ops per second."""
    a = torch.randint(-3, 4, (size, size), dtype=torch.int8, device="cuda")
    b = torch.randint(-3, 4, (size, size), dtype=torch.int8, device="cuda")
    for _ in range(3):
        torch._int_mm(a, b)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(reps):
        torch._int_mm(a, b)
    stop.record()
    torch.cuda.synchronize()
    return 2.0 * size ** 3 * reps / (start.elapsed_time(stop) * 1e-3) / 1e12


def main() -> None:
    import torch

    props = torch.cuda.get_device_properties(0)
    l2 = []
    for mib in (16, 32, 48):
        gbs = copy_gbs(torch, mib << 20, 500, graph=True)
        l2.append(gbs)
        print(json.dumps({"buffer_pair_mib": 2 * mib, "copy_gbs": round(gbs, 1), "resident": "L2"}))
    hbm = copy_gbs(torch, 2 << 30, 20)
    print(json.dumps({"buffer_pair_mib": 4096, "copy_gbs": round(hbm, 1), "resident": "HBM"}))
    print(f"device: {props.name}, {props.multi_processor_count} SMs, L2 {props.L2_cache_size >> 20} MiB")
    tops = int8_tops(torch, 8192, 50)
    print(json.dumps({"gemm": "int8 8192^3 (torch._int_mm)", "tops": round(tops, 1)}))
    print(f"l2_copy_gbs: {max(l2):.1f}")
    print(f"hbm_copy_gbs: {hbm:.1f}")
    print(f"int8_tops: {tops:.1f}")


if __name__ == "__main__":
    main()
