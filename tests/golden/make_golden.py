"""Regenerates the golden fixtures in tests/golden/ (run in a container that has the reference checkout).

Two kinds of fixtures:

* ``published.json`` — rows of the reference's published result tables, read as data from its
  ``docs/data/*.csv``.  Every row is a full PBILS run on the CPU and GPU backends of the reference
  with the protocol its scripts used (``docs/gpu_sweep.sh:13-15``, ``docs/gww_sweep.py:38-103``,
  ``docs/benchmarks.md:56-62``), so the row's ``f`` (and, where given, ``iters``) pins the trajectory.
* ``reference_runs.json`` — outputs of the reference's own CPU code (``oracle/_ref/libccref.so``,
  built by ``oracle/Makefile`` from the reference sources) on small seeded cases: PBILS with varied
  parameters (labels included), Neighborhood on every graph with n <= 4 and on the Erdős–Rényi set of
  ``cuda/cc_verify_gpu.cu:88-112``.

Usage:  python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import csv
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

from oracle import Reference, make_params  # noqa: E402


def published(ref_root: str) -> dict:
    data = os.path.join(ref_root, "docs", "data")
    out = {"gpu_csv": [], "gww_stop_csv": [], "cpu_csv": [], "gww_csv": []}
    # gpu.csv: --density 0.33 --graph-seed 7 --iters 20 --early-stop 1000 --gww 0, seed = 5 + run
    with open(os.path.join(data, "gpu.csv")) as fh:
        for line_no, row in enumerate(csv.DictReader(fh), start=2):
            out["gpu_csv"].append({"line": line_no, "n": int(row["n"]), "k": int(row["k"]), "pop": int(row["pop"]),
                                   "seed": 5 + int(row["run"]), "f": int(row["gpu_f"]), "cpu_f": int(row["cpu_f"])})
    # gww_stop.csv: --density 0.33 --graph-seed g --seed 1 --runs 9 (run r -> seed r + 1), default
    # --iters 100 and --early-stop 6; rows of the 'random' set only (the real graphs are not here)
    with open(os.path.join(data, "gww_stop.csv")) as fh:
        for line_no, row in enumerate(csv.DictReader(fh), start=2):
            if row["set"] != "random":
                continue
            out["gww_stop_csv"].append({"line": line_no, "graph_seed": int(row["graph"].split("_")[1]),
                                        "n": int(row["n"]), "k": int(row["k"]), "pop": int(row["pop"]),
                                        "gww": float(row["gww"]), "seed": int(row["seed"]), "f": int(row["f"]),
                                        "iters": int(row["iters"])})
    # cpu.csv 'ours_*' rows: 5 iterations, gww 0, seeds 5 + rep, graph-seed 7, density 0.33
    with open(os.path.join(data, "cpu.csv")) as fh:
        for line_no, row in enumerate(csv.DictReader(fh), start=2):
            if not row["variant"].startswith("ours"):
                continue
            out["cpu_csv"].append({"line": line_no, "n": int(row["n"]), "k": int(row["k"]), "pop": int(row["pop"]),
                                   "seed": 5 + int(row["rep"]), "f": int(row["f"]),
                                   "threads": int(row["variant"].split("_")[1])})
    # gww.csv: record at checkpoint iterations of long runs without early stop (--iters = --early-stop);
    # random set, seed = run + 1.  Kept for n = 1000 (short GPU runs).
    with open(os.path.join(data, "gww.csv")) as fh:
        runs: dict = {}
        for line_no, row in enumerate(csv.DictReader(fh), start=2):
            if row["set"] != "random" or int(row["n"]) != 1000:
                continue
            key = (row["graph"], int(row["k"]), int(row["pop"]), row["gww"], int(row["seed"]))
            runs.setdefault(key, []).append((int(row["iter"]), int(row["record"]), line_no))
        for (graph, k, pop, gww, seed), pts in sorted(runs.items()):
            out["gww_csv"].append({"graph_seed": int(graph.split("_")[1]), "n": 1000, "k": k, "pop": pop,
                                   "gww": float(gww), "seed": seed, "iters": max(p[0] for p in pts),
                                   "checkpoints": [[p[0], p[1]] for p in pts], "first_line": pts[0][2]})
    return out


def graph_from_pairs(n: int, mask: int) -> np.ndarray:
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


def reference_runs() -> dict:
    ref = Reference()
    pbils = []
    cases = [
        # n, density, graph_seed, k, pop, tournament, iterations, early_stop, perturbation, gww, seed
        (1, 0.5, 1, 2, 4, 5, 3, 6, 0.4, 0.1, 1),
        (2, 1.0, 2, 2, 3, 2, 4, 6, 0.4, 0.0, 2),
        (7, 0.5, 3, 3, 5, 3, 6, 6, 0.4, 0.2, 3),
        (31, 0.3, 4, 2, 16, 5, 10, 3, 0.4, 0.1, 4),
        (32, 0.5, 5, 4, 16, 5, 10, 4, 0.3, 0.25, 5),
        (33, 0.7, 6, 5, 16, 5, 10, 10, 0.5, 0.5, 6),
        (64, 0.2, 7, 1, 8, 5, 5, 6, 0.4, 0.1, 7),
        (65, 0.5, 8, 7, 12, 1, 8, 8, 0.0, 0.1, 8),
        (100, 0.45, 9, 3, 20, 4, 12, 12, 0.6, 0.1, 9),
        (127, 0.1, 10, 9, 24, 5, 6, 2, 0.4, 0.0, 10),
        (129, 0.9, 11, 2, 10, 3, 8, 0, 0.4, 0.1, 11),
        (200, 0.33, 12, 16, 32, 5, 5, 6, 0.4, 0.1, 12),
        (257, 0.5, 13, 33, 8, 5, 4, 6, 0.4, 0.1, 13),
        (300, 0.5, 14, 64, 6, 5, 3, 6, 0.4, 0.2, 14),
        (150, 0.4, 99, 3, 24, 5, 15, 15, 0.4, 0.25, 1),
        (500, 0.33, 7, 2, 128, 5, 5, 6, 0.4, 0.0, 5),
    ]
    for (n, density, gseed, k, pop, tour, iters, early, pert, gww, seed) in cases:
        bits, edges = ref.erdos_renyi(n, density, gseed)
        p = make_params(k=k, population=pop, tournament=tour, iterations=iters, early_stop=early,
                        perturbation=pert, gww=gww, seed=seed)
        sol = ref.pbils(bits, p, threads=4)
        pbils.append({"n": n, "density": density, "graph_seed": gseed, "edges": edges, "k": k, "population": pop,
                      "tournament": tour, "iterations": iters, "early_stop": early, "perturbation": pert,
                      "gww": gww, "seed": seed, "objective": sol.objective, "iterations_done": sol.iterations_done,
                      "clusters_used": sol.clusters_used, "local_searches": sol.local_searches,
                      "accepted_moves": sol.accepted_moves, "labels": sol.labels.tolist()})

    neighborhood = []
    for n in range(1, 5):
        pairs = n * (n - 1) // 2
        for mask in range(1 << pairs):
            bits = graph_from_pairs(n, mask)
            entry = {"n": n, "mask": mask}
            for ls in (False, True):
                sol = ref.neighborhood(bits, ls)
                entry["ls" if ls else "plain"] = {"objective": sol.objective, "labels": sol.labels.tolist(),
                                                  "accepted_moves": sol.accepted_moves,
                                                  "clusters_used": sol.clusters_used}
            neighborhood.append(entry)
    for n in (31, 32, 33, 127, 129, 257):
        for density in (0.0, 0.2, 0.5, 1.0):
            bits, edges = ref.erdos_renyi(n, density, 19 + n)
            entry = {"n": n, "density": density, "graph_seed": 19 + n, "edges": edges}
            for ls in (False, True):
                sol = ref.neighborhood(bits, ls)
                entry["ls" if ls else "plain"] = {"objective": sol.objective, "labels": sol.labels.tolist(),
                                                  "accepted_moves": sol.accepted_moves,
                                                  "clusters_used": sol.clusters_used}
            neighborhood.append(entry)
    return {"pbils": pbils, "neighborhood": neighborhood}


def main() -> None:
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    with open(os.path.join(HERE, "published.json"), "w") as fh:
        json.dump(published(ref_root), fh, separators=(",", ":"))
    with open(os.path.join(HERE, "reference_runs.json"), "w") as fh:
        json.dump(reference_runs(), fh, separators=(",", ":"))


if __name__ == "__main__":
    main()
