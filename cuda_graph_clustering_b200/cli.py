"""``cc_gpu`` command line on the B200 solver: the reference's CLI flags, output lines, result JSON and exit
codes (include/cc_cli.hpp:124-183 flags, :284-377 Main, :248-277 WriteResultJson), over this package.

    python -m cuda_graph_clustering_b200.cli --n 1000 --density 0.5 --k 5 --pop 128 --iters 100

Instances: a seeded G(n, p) (``Graph::ErdosRenyi``, generated on the device bit-exactly) or an edge list
(``--edges``: ``Graph::LoadEdgeList``, src/cc_graph.cpp:270-306 -- any integer ids, a vertex is the rank of its
id, ``#`` / ``%`` comment lines and lines not starting with a number are skipped, self-loops dropped) or a tags
file (``--tags``: ``Graph::LoadTags``, src/cc_graph.cpp:311-371, built on the device).  The
post-solve check recounts the objective on the GPU over the bit rows (``ccb_evaluate_labelings``, the
reference's ``ObjectiveBitwise``); a mismatch exits 2, any error prints ``error: ...`` and exits 1.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

ALGORITHMS = ("pbils", "NeighborhoodCuda", "NeighborhoodWithManyLocalSearchesCuda")
# the names the reference prints and writes (AlgorithmName, include/cc_cli.hpp:22-28)
ALGORITHM_NAMES = {"pbils": "PBILS", "NeighborhoodCuda": "NeighborhoodCuda",
                   "NeighborhoodWithManyLocalSearchesCuda": "NeighborhoodWithManyLocalSearchesCuda"}
LS_KERNELS = {"auto": 0, "global": 1, "shared": 2, "wide": 3}


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="cc_gpu", description="PBILS k-correlation clustering on the GPU")
    g = ap.add_argument_group("instance")
    g.add_argument("--n", type=int, default=500, help="generate G(n, p) on N vertices")
    g.add_argument("--density", type=float, default=0.5, help="edge probability")
    g.add_argument("--graph-seed", type=int, default=1, help="generator seed, fixes the instance")
    g.add_argument("--edges", default="", help="load an edge list (SNAP, CSV): any ids, a vertex is their rank")
    g.add_argument("--tags", default="", help="graph by tags ({\"key\": [\"tag\", ...]} JSON): n random objects "
                                              "by --graph-seed, joined when --similarity >= --threshold")
    g.add_argument("--similarity", default="jaccard", help="measure for --tags: jaccard, cosine, dice, overlap")
    g.add_argument("--threshold", type=float, default=0.5, help="threshold for --tags")
    a = ap.add_argument_group("algorithm")
    a.add_argument("--algorithm", choices=ALGORITHMS, default="pbils")
    a.add_argument("--k", type=int, default=2, help="upper bound on the number of clusters")
    a.add_argument("--pop", type=int, default=128, help="population; for Neighborhood: partitions per batch")
    a.add_argument("--tournament", type=int, default=5)
    a.add_argument("--iters", type=int, default=100)
    a.add_argument("--early-stop", type=int, default=6)
    a.add_argument("--perturb", type=float, default=0.4)
    a.add_argument("--gww", type=float, default=0.1)
    a.add_argument("--seed", type=int, default=1)
    a.add_argument("--threads", type=int, default=1, help="CPU only (accepted and ignored)")
    a.add_argument("--time-limit", type=float, default=0.0)
    a.add_argument("--ls-kernel", choices=tuple(LS_KERNELS), default="auto")
    e = ap.add_argument_group("experiment")
    e.add_argument("--runs", type=int, default=1)
    e.add_argument("--no-verify", dest="verify", action="store_false")
    e.add_argument("--out", default="", help="write the result as JSON")
    e.add_argument("--labels-out", default="", help="write the best clustering as labels")
    e.add_argument("--verbose", action="store_true")
    return ap


def load_edge_list(path: str):
    """Graph::LoadEdgeList (src/cc_graph.cpp:270-306)."""
    import cuda_graph_clustering_b200 as ccb

    ends = []
    with open(path, "rb") as f:
        for raw in f:
            line = raw.decode("latin-1")
            if not line or line[0] in "#%":
                continue
            pos, ids = 0, []
            for _ in range(2):
                while pos < len(line) and line[pos] in " \t,":
                    pos += 1
                start = pos
                while pos < len(line) and line[pos].isdigit():
                    pos += 1
                if pos == start:
                    break
                value = int(line[start:pos])
                if value >= 1 << 64:
                    raise RuntimeError(f"vertex id does not fit 64 bits in {path}")
                ids.append(value)
            if len(ids) == 2:
                ends.extend(ids)
    if not ends:
        raise RuntimeError(f"no edges in {path}")
    arr = np.array(ends, dtype=np.uint64)
    uniq = np.unique(arr)
    if uniq.size >= 1 << 32:
        raise RuntimeError(f"too many vertices in {path}")
    rank = np.searchsorted(uniq, arr).astype(np.int64).reshape(-1, 2)
    n = int(uniq.size)
    bits = np.zeros((n, ccb.words_per_row(n)), np.uint32)
    u, v = rank[:, 0], rank[:, 1]
    keep = u != v
    u, v = u[keep], v[keep]
    np.bitwise_or.at(bits, (u, v // 32), np.uint32(1) << (v % 32).astype(np.uint32))
    np.bitwise_or.at(bits, (v, u // 32), np.uint32(1) << (u % 32).astype(np.uint32))
    edges = int(sum(int(x).bit_count() for x in bits.ravel())) // 2
    return ccb.Graph(n, bits, edges)


def recount(graph, labels: np.ndarray, k: int) -> int:
    """The objective of `labels` recounted on the GPU over the bit rows (ccb_evaluate_labelings)."""
    import torch

    import cuda_graph_clustering_b200 as ccb

    n = graph.n
    if n == 0:
        return 0
    bits = torch.from_numpy(np.ascontiguousarray(graph.bits)).cuda()
    lab = torch.from_numpy(labels.astype(np.int32)).cuda()
    f = torch.zeros(1, dtype=torch.int64, device="cuda")
    ccb.evaluate_labelings(bits.data_ptr(), n, graph.WordsPerRow(), graph.edges, k, 1, lab.data_ptr(),
                           f.data_ptr())
    torch.cuda.synchronize()
    return int(f.item())


def write_result_json(path, graph, args, best, avg_objective, worst, avg_seconds):
    """WriteResultJson (include/cc_cli.hpp:248-277): the same keys in the same order."""
    lines = ["{",
             f'  "algorithm": "{ALGORITHM_NAMES[args.algorithm]}",',
             '  "backend": "gpu",',
             f'  "size": {graph.n},',
             f'  "edges": {graph.edges},',
             f'  "density": {graph.Density():g},',
             f'  "k": {args.k},',
             f'  "population": {args.pop},',
             f'  "gww": {args.gww:g},',
             f'  "runs": {args.runs},',
             f'  "objective function value": {best.objective},',
             f'  "objective average": {avg_objective:g},',
             f'  "objective max": {worst},',
             f'  "computation time seconds": {best.seconds:g},',
             f'  "computation time average": {avg_seconds:g},',
             f'  "clusters used": {best.clusters_used},',
             '  "clustering vector": [' + ",".join(str(int(x)) for x in best.labels) + "]",
             "}"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None) -> int:
    args = parser().parse_args(argv)
    import cuda_graph_clustering_b200 as ccb

    try:
        if args.tags:  # Graph::LoadTags (src/cc_graph.cpp:311-371), built on the device
            graph = ccb.DeviceGraph.load_tags(args.tags, args.similarity, args.threshold, args.n,
                                              args.graph_seed).download()
        elif args.edges:
            graph = load_edge_list(args.edges)
        else:
            graph = ccb.DeviceGraph.erdos_renyi(args.n, args.density, args.graph_seed).download()
    except Exception as error:  # the reference prints the loader's message and exits 1
        print(f"error: {error}")
        return 1
    print("backend      gpu")
    print(f"instance     n={graph.n}  edges={graph.edges}  density={graph.Density():.4f}")
    if args.algorithm == "pbils":
        print(f"algorithm    PBILS  k={args.k}  pop={args.pop}  tournament={args.tournament}  iters={args.iters}  "
              f"early-stop={args.early_stop}  perturb={args.perturb:.2f}  gww={args.gww:.2f}")
        solve = ccb.SolveGpu
    else:
        print(f"algorithm    {args.algorithm}  k={args.k}  batch={args.pop}")
        solve = ccb.SolveNeighborhoodGpu if args.algorithm == "NeighborhoodCuda" else \
            ccb.SolveNeighborhoodWithManyLocalSearchesGpu
    best, worst, f_sum, s_sum = None, 0, 0.0, 0.0
    for run in range(args.runs):
        params = ccb.PbilsParams(k=args.k, population=args.pop, tournament=args.tournament, iterations=args.iters,
                                 early_stop=args.early_stop, perturbation=args.perturb, gww=args.gww,
                                 threads=args.threads, seed=args.seed + run, time_limit_sec=args.time_limit,
                                 verbose=args.verbose, ls_kernel=LS_KERNELS[args.ls_kernel])
        try:
            result = solve(graph, params)
        except Exception as error:
            print(f"error: {error}")
            return 1
        if args.verify:
            truth = recount(graph, np.asarray(result.labels), args.k)
            if truth != result.objective:
                print(f"MISMATCH run {run}: reported {result.objective}, recount {truth}")
                return 2
        f_sum += result.objective
        s_sum += result.seconds
        if best is None or result.objective < best.objective:
            best = result
        if run == 0 or result.objective > worst:
            worst = result.objective
        print(f"run {run:<3d}      f={result.objective:<10d}  clusters={result.clusters_used:<3d}  "
              f"iters={result.iterations_done:<4d}  {result.seconds:.3f}s")
        if args.verbose and result.local_searches > 0:
            print(f"moves        {result.accepted_moves} accepted, "
                  f"{result.accepted_moves / result.local_searches:.0f} per local search")
    avg_f, avg_s = f_sum / args.runs, s_sum / args.runs
    print("---")
    print(f"objective    min={best.objective}  avg={avg_f:.2f}  max={worst}")
    print(f"time         best={best.seconds:.3f}s  avg={avg_s:.3f}s")
    if args.verify:
        print("verified     reported value recounted over bit rows on the GPU")
    if args.out:
        write_result_json(args.out, graph, args, best, avg_f, worst, avg_s)
        print(f"written      {args.out}")
    if args.labels_out:
        with open(args.labels_out, "w") as f:
            f.write(" ".join(str(int(x)) for x in best.labels) + "\n")
        print(f"written      {args.labels_out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
