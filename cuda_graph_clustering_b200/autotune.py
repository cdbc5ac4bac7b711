"""Autotuner of the batched engine: per shape class, the descent kernel, threads per slot and resident block
count that give the most solves per second.

    python -m cuda_graph_clustering_b200.autotune [--out PATH] [--instances N] [--iterations I]

A shape class is a range of n and k that the planner maps to one batched kernel family (incremental with
cached keys, incremental with its state in global memory, streamed packed k <= 8).  For each class the tuner
draws seeded planted instances with the batched mix's parameters (communities 2..16, p_in [0.3, 0.8], p_out
[0.01, 0.2], flips [0.05, 0.2], population {32, 64, 128}) restricted to the class's n and k, solves them as
one batch under every candidate setting (installed with ccb_tuning_set), checks that every candidate gives
the same objectives, and keeps the fastest.  The table is written as JSON (``tuning.json`` beside this
module is the committed one, loaded by Batch and Server on first use).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import cuda_graph_clustering_b200 as ccb
from cuda_graph_clustering_b200.workloads import Draws

# kind codes of ccb_tuning_entry
REGISTERS, STREAM, INCREMENTAL, INCREMENTAL_REGS = 0, 1, 2, 3

# (name, plan kind, n_min, n_max, k_min, k_max, candidates); a candidate is (use_kind, threads, blocks_per_sm,
# max_slots) with use_kind -1 = the plan's kernel.
GLOBAL_FORMS = [(INCREMENTAL, 256, 0, 0), (INCREMENTAL, 512, 0, 0), (INCREMENTAL, 1024, 0, 0)]
CLASSES = [
    ("incremental, cached keys, 8192 < n <= 16384", INCREMENTAL_REGS, 8193, 16384, 9, 64,
     [(-1, 0, 0, 0)] + GLOBAL_FORMS),
    ("incremental, cached keys, 4096 < n <= 8192", INCREMENTAL_REGS, 4097, 8192, 9, 64,
     [(-1, 0, 0, 0)] + GLOBAL_FORMS),
    ("incremental, cached keys, 2048 < n <= 4096", INCREMENTAL_REGS, 2049, 4096, 9, 64,
     [(-1, 0, 0, 0)] + GLOBAL_FORMS),
    ("incremental, global state, 16384 < n <= 32767", INCREMENTAL, 16385, 32767, 9, 64,
     [(-1, 0, 0, 0)] + GLOBAL_FORMS[:2]),
    ("streamed packed k <= 8, 4096 < n <= 32767", STREAM, 4097, 32767, 2, 8,
     [(-1, 0, 0, 0), (-1, 0, 1, 0), (-1, 0, 0, 148)]),
]


def class_instances(n_min, n_max, k_min, k_max, count, seed, iterations):
    d = Draws(seed, 0x7A7E)
    out = []
    for _ in range(count):
        n = int(round(math.exp(math.log(n_min) + d.unit() * math.log(n_max / n_min))))
        parts = 2 + d.below(15)
        p_in = 0.3 + 0.5 * d.unit()
        p_out = 0.01 + 0.19 * d.unit()
        flip = 0.05 + 0.15 * d.unit()
        k = k_min + d.below(k_max - k_min + 1)
        pop = (32, 64, 128)[d.below(3)]
        g, _ = ccb.DeviceGraph.planted(n, parts, p_in, p_out, flip, d.u64())
        out.append((g, ccb.PbilsParams(k=k, population=pop, iterations=iterations, early_stop=iterations,
                                       gww=0.1, seed=d.u64())))
    return out


def entry(kind, n_min, n_max, k_min, k_max, cand):
    use_kind, threads, bps, cap = cand
    return dict(kind=kind, n_min=n_min, n_max=n_max, k_min=k_min, k_max=k_max, use_kind=use_kind,
                threads=threads, blocks_per_sm=bps, max_slots=cap)


def time_batch(instances):
    b = ccb.Batch()
    for g, p in instances:
        b.add(g, p)
    t0 = time.perf_counter()
    b.run()
    dt = time.perf_counter() - t0
    objectives = [b.result(i).objective for i in range(len(instances))]
    desc = b.describe()
    b.close()
    return dt, objectives, desc


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=ccb.TUNING_PATH)
    ap.add_argument("--instances", type=int, default=32)
    ap.add_argument("--iterations", type=int, default=4)
    ap.add_argument("--seed", type=int, default=5)
    args = ap.parse_args()
    import torch

    torch.cuda.set_device(0)
    ccb.load_tuning("/nonexistent")  # start from the planner's defaults
    entries, report = [], []
    for ci, (name, kind, n_min, n_max, k_min, k_max, cands) in enumerate(CLASSES):
        inst = class_instances(n_min, n_max, k_min, k_max, args.instances, args.seed + ci, args.iterations)
        ccb.set_tuning([])
        time_batch(inst[:2])  # module load and first-launch costs
        best, base_obj, rows = None, None, []
        for cand in cands:
            ccb.set_tuning([entry(kind, n_min, n_max, k_min, k_max, cand)])
            dt, obj, desc = time_batch(inst)
            if base_obj is None:
                base_obj = obj
            if obj != base_obj:
                raise RuntimeError(f"{name}: candidate {cand} changed a result")
            rows.append(dict(candidate=entry(kind, n_min, n_max, k_min, k_max, cand), seconds=dt,
                             solves_per_s=len(inst) / dt, buckets=desc))
            print(json.dumps(dict(cls=name, candidate=cand, seconds=round(dt, 4))), flush=True)
            if best is None or dt < best[1]:
                best = (cand, dt)
        entries.append(entry(kind, n_min, n_max, k_min, k_max, best[0]))
        report.append(dict(cls=name, instances=len(inst), iterations=args.iterations, best=best[0],
                           speedup_vs_plan=rows[0]["seconds"] / best[1], rows=rows))
        for g, _ in inst:
            g.close()
    ccb.set_tuning([])
    props = torch.cuda.get_device_properties(0)
    with open(args.out, "w") as f:
        json.dump(dict(device=props.name, sms=props.multi_processor_count, entries=entries,
                       measurements=report), f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
