"""Benchmark of the PBILS hot path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload plain]

Workload "plain": the reference's plain PBILS configuration, G(n=1000, p=0.5) from graph seed 1,
k=5, population 128, tournament 5, perturbation 0.4, gww 0.1, 100 iterations with the early stop
disabled (--early-stop 100), search seed 1 (rank r uses seed 1 + r).  One step = one full solve.
Metric: PBILS iterations per second over the whole job (all ranks), plus LS moves/s.

`value`: device time (CUDA events on the solver's stream) of solves on a graph and buffers already
resident in HBM; L2 is flushed (a 256 MiB write) between timed steps, outside the events.
`e2e`: the one-call public C ABI (ccb_pbils_solve) from a pinned host bitset to host labels, wall
clock, every step paying the bitset upload, the degree count and the label read-back (the library keeps
its device buffers across one-call solves of the same shape, so only the first call allocates).
Every step's objective is checked against the value the CPU oracle gives for this instance.

Other workloads: large (G(32000, 0.33), k=8), wide2 / wide3 (G(65536, 0.02), k=2 / 3), batched (the
256-instance mix, batched engine vs plain path), serving (Poisson request stream, server vs plain FIFO).

Multi-GPU (torchrun): each rank solves its own instance (a different search seed) with no
collective on the data path ("scaling": "weak"); the only collectives are the timing barrier, the
max over ranks of the times and the sum of the counts (combine_over_ranks).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

PLAIN = dict(n=1000, density=0.5, graph_seed=1, k=5, population=128, tournament=5, perturbation=0.4, gww=0.1,
             iterations=100, early_stop=100, seed=1)
PLAIN_OBJECTIVE = {1: 234911}  # seed -> objective of the CPU oracle (and the reference binary)
# The large plain configuration of the hot-path roofline target: G(32000, 0.33) from graph seed 7, k=8,
# pop 128; a step is a short solve (3 iterations) because one iteration costs ~10^4 moves per slot.
LARGE = dict(n=32000, density=0.33, graph_seed=7, k=8, population=128, tournament=5, perturbation=0.4, gww=0.1,
             iterations=3, early_stop=100, seed=1)
# The wide configuration: G(65536, 0.02) (a 512 MiB bitset) from graph seed 1, k = 2 or 3 on the packed wide
# descents (int32 G), pop 128, gww 0.1, 50 iterations.  No CPU objective is known at this size: every step's
# labels are recounted on the GPU instead (ccb_evaluate_labelings) and must give the reported objective.
WIDE2 = dict(n=65536, density=0.02, graph_seed=1, k=2, population=128, tournament=5, perturbation=0.4, gww=0.1,
             iterations=50, early_stop=50, seed=1)
WIDE3 = dict(WIDE2, k=3)
# The published docs/data/gpu.csv row at the narrow limit (line 26): ER(32000, 0.33, graph seed 7), k=3, pop 128,
# 20 iterations, gww 0, early stop off, seed 6 -> f = 224579124 (GPU and CPU alike).
GPUCSV32K = dict(n=32000, density=0.33, graph_seed=7, k=3, population=128, tournament=5, perturbation=0.4, gww=0.0,
                 iterations=20, early_stop=1000, seed=6)
WORKLOADS = {"plain": (PLAIN, PLAIN_OBJECTIVE), "large": (LARGE, {}), "wide2": (WIDE2, {}), "wide3": (WIDE3, {}),
             "gpucsv32k": (GPUCSV32K, {6: 224579124})}
# The Neighborhood configuration: the planted two-community graph, n = 4096 split 2048/2048 by a seeded
# permutation, p_in 0.6, p_out 0.1 (graph seed 1), batches of 128 start partitions (32 full batches).
NEIGHBORHOOD = dict(n=4096, parts=2, shuffle_split=True, p_in=0.6, p_out=0.1, flip=0.0, graph_seed=1, batch=128)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched", "serving", "neighborhood"],
                    default="plain")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rebuild", choices=["auto", "popcount", "tensor"], default="auto",
                    help="wide workloads: how G = A*Z is rebuilt (the tensor path is timed beside the popcount one)")
    ap.add_argument("--batch-count", type=int, default=256, help="batched workload: instances")
    ap.add_argument("--batch-iters", type=int, default=100, help="batched workload: iterations per instance")
    ap.add_argument("--batch-engine", choices=["flow", "lockstep"], default="lockstep",
                    help="batched workload: engine")
    ap.add_argument("--serve-count", type=int, default=32, help="serving workload: requests")
    ap.add_argument("--serve-rate", type=float, default=10.0, help="serving workload: Poisson arrivals per second")
    ap.add_argument("--serve-max-n", type=int, default=32767,
                    help="serving workload: largest n (the full stream goes to 50000; requests beyond 32767 run "
                         "on side threads and take tens of seconds each, so the default sample stops there)")
    ap.add_argument("--serve-budget-gb", type=float, default=0.0, help="serving workload: HBM budget (0: 80%% free)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    """HBM copy GB/s: the pool's MEASURED_PEAKS.json when present, else this repository's own measurement on the
    same B200s (profiles/peaks_l2_hbm_int8.txt), else the 6650 GB/s recipe fallback."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        pass
    own = profiled_value("peaks_l2_hbm_int8", "hbm_copy_gbs")
    if own:
        return own, "measured (profiles/peaks_l2_hbm_int8.txt)"
    return 6650.0, "fallback"


def profiled_value(name: str, key: str):
    """A `key: value` figure from a committed summary under profiles/ (name without .txt), or None."""
    path = os.path.join(REPO, "profiles", name + ".txt")
    try:
        with open(path) as fh:
            m = re.search(re.escape(key) + r":\s*([0-9.eE+]+)", fh.read())
            return float(m.group(1)) if m else None
    except OSError:
        return None


def profiled_traffic(name: str):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>.txt), or None."""
    return profiled_value(name, "dram_bytes_per_launch")


def measured_peaks():
    """L2 copy GB/s and int8 tensor TOPS measured on this pool (profiles/peaks_l2_hbm_int8.txt, written by
    cuda_graph_clustering_b200/peaks.py)."""
    return profiled_value("peaks_l2_hbm_int8", "l2_copy_gbs"), profiled_value("peaks_l2_hbm_int8", "int8_tops")


def reference_cpu_run(cfg, iterations, threads=0):
    """One run of the reference's own CPU binary (oracle/_ref/cc_cpu); returns (solver seconds, f)."""
    exe = os.path.join(REPO, "oracle", "_ref", "cc_cpu")
    cmd = [exe, "--n", str(cfg["n"]), "--density", str(cfg["density"]), "--graph-seed", str(cfg["graph_seed"]),
           "--k", str(cfg["k"]), "--pop", str(cfg["population"]), "--tournament", str(cfg["tournament"]),
           "--perturb", str(cfg["perturbation"]), "--gww", str(cfg["gww"]), "--iters", str(iterations),
           "--early-stop", str(cfg["early_stop"]), "--seed", str(cfg["seed"]), "--threads", str(threads),
           "--no-verify"]
    out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
    t = float(re.search(r"time\s+best=([0-9.]+)s", out).group(1))
    f = int(re.search(r"objective\s+min=(\d+)", out).group(1))
    threads_used = int(re.search(r"threads\s+(\d+)", out).group(1))
    return t, f, threads_used


def reference_gpu_run(cfg, runs=3):
    """The reference's own GPU binary (oracle/_ref/cc_gpu_ref: its CUDA sources compiled for sm_100a) on the same
    instance: (best solver seconds over `runs` runs of seeds seed .. seed + runs - 1, objective of the run with
    this seed), or None when it was not built.  The first run also pays the CUDA context set-up."""
    exe = os.path.join(REPO, "oracle", "_ref", "cc_gpu_ref")
    if not os.path.exists(exe):
        return None
    cmd = [exe, "--n", str(cfg["n"]), "--density", str(cfg["density"]), "--graph-seed", str(cfg["graph_seed"]),
           "--k", str(cfg["k"]), "--pop", str(cfg["population"]), "--tournament", str(cfg["tournament"]),
           "--perturb", str(cfg["perturbation"]), "--gww", str(cfg["gww"]), "--iters", str(cfg["iterations"]),
           "--early-stop", str(cfg["early_stop"]), "--seed", str(cfg["seed"]), "--runs", str(runs), "--no-verify"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, check=True).stdout
    # run r uses seed + r and the same fixed iteration count; run 0 has this instance's seed
    t = float(re.search(r"time\s+best=([0-9.]+)s", out).group(1))
    f = int(re.search(r"run 0\s+f=(\d+)", out).group(1))
    return t, f


def workload_text(name, cfg):
    """The `config.workload` string of a PBILS workload, shared by both arms."""
    return (f"{name} PBILS: ER(n={cfg['n']}, p={cfg['density']}, graph seed {cfg['graph_seed']}), k={cfg['k']}, "
            f"pop={cfg['population']}, tournament 5, perturb 0.4, gww 0.1, {cfg['iterations']} iterations "
            f"(early stop off), seed {cfg['seed']} + rank")


def run_reference(args, rank):
    """--impl reference: the reference's CPU implementation on this box's host cores."""
    if rank != 0:
        return
    cfg = dict(PLAIN)
    sample_iters = 10
    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "cc_cpu")):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cc_cpu not built"}))
        return
    for _ in range(args.warmup):
        reference_cpu_run(cfg, 2)
    total_t, total_it, threads = 0.0, 0, 0
    for _ in range(args.steps):
        t, f, threads = reference_cpu_run(cfg, sample_iters)
        total_t += t
        total_it += sample_iters
    value = total_it / total_t
    line = {"metric": "PBILS iter/s", "value": value, "unit": "iter/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_text("plain", cfg),
                       "sample": f"{sample_iters} iterations per step (of 100)", "parallelism": "replicas x1"},
            "cpu_baseline": {"value": value, "unit": "iter/s", "cores": threads, "kind": "reference",
                             "sample": f"{sample_iters} of the 100 iterations, --threads 0"},
            "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def combine_over_ranks(dist, maxes, sums, device="cuda"):
    """The replicas' only collectives: the max over ranks of the times, the sum over ranks of the counts.
    Returns (maxes, sums) as lists of floats; without a process group the inputs come back unchanged."""
    import torch

    if dist is None:
        return [float(x) for x in maxes], [float(x) for x in sums]
    mx = torch.tensor([float(x) for x in maxes], dtype=torch.float64, device=device)
    sm = torch.tensor([float(x) for x in sums], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


def percentile(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(math.ceil(q * len(xs))) - 1)] if xs else None


def run_batched(args, rank, world, local):
    """The batched mix (cuda_graph_clustering_b200.workloads.batched_mix, master seed 7 + rank): every
    instance solved by the batched engine (all together, one graph replay per iteration) and by the plain
    path (one ccb_solver_pbils call per instance, in order), on the same device-resident graphs; each
    batched result is checked equal to its plain result.  Latencies are completion times of a FIFO in
    which all instances arrive at once."""
    import torch

    import cuda_graph_clustering_b200 as ccb
    from cuda_graph_clustering_b200.workloads import batched_mix

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    mix = batched_mix(args.batch_count, master=7 + rank, iterations=args.batch_iters)
    graphs = [ccb.DeviceGraph.planted(i.n, i.parts, i.p_in, i.p_out, i.flip, i.graph_seed)[0] for i in mix]
    params = [ccb.PbilsParams(k=i.k, population=i.population, iterations=i.iterations, early_stop=i.iterations,
                              gww=0.1, seed=i.seed) for i in mix]
    batch = ccb.Batch(engine=args.batch_engine)
    ids = [batch.add(g, p) for g, p in zip(graphs, params)]
    # warm-up: one iteration of a batch of every instance shape (module loading, first launches, graph
    # instantiation paths), not the timed batch itself, whose run takes minutes
    warm = ccb.Batch(engine=args.batch_engine)
    for g, i in zip(graphs, mix):
        warm.add(g, ccb.PbilsParams(k=i.k, population=i.population, iterations=1, early_stop=1, gww=0.1,
                                    seed=i.seed + 1))

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        warm.run()
    warm.close()
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_batch = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        batch.run()
        t_batch.append(time.perf_counter() - t0)
    clock_info = clocks.stop()
    got = [batch.result(i) for i in ids]

    solvers = [ccb.Solver(g, p) for g, p in zip(graphs, params)]
    for s_, p in list(zip(solvers, params))[:8]:
        s_.pbils(p, want_labels=False)
    torch.cuda.synchronize()
    t_plain = []
    exact = True
    for s_, p, r in zip(solvers, params, got):
        t0 = time.perf_counter()
        w = s_.pbils(p)
        t_plain.append(time.perf_counter() - t0)
        exact &= (w.objective == r.objective and w.iterations_done == r.iterations_done
                  and w.accepted_moves == r.accepted_moves and bool((w.labels == r.labels).all()))
    barrier()
    tb = max(t_batch)
    tp = sum(t_plain)
    (tb_all, tp_all), _ = combine_over_ranks(dist, [tb, tp], [])
    if rank == 0:
        count = len(mix)
        done = []
        acc = 0.0
        for t in t_plain:
            acc += t
            done.append(acc)
        # each instance's own completion time in the batch (the flow engine reports it; the lock-step engine
        # finishes every instance of equal iteration count at the run's end)
        own = sorted(r.seconds for r in got) if args.batch_engine == "flow" else [tb] * count
        # the most batching can give at one running slot per SM: the plain path runs an instance's slots side by
        # side (all iterations of instance i take t_i, pop_i of the SMs busy), so the batch needs at least
        # sum_i pop_i t_i / SMs and at least the longest t_i
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        packed = max(max(t_plain), sum(m.population * t for m, t in zip(mix, t_plain)) / sms)
        line = {
            "metric": "batched solves/s", "value": world * count / tb_all, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tb_all, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
            "config": {"workload": f"batched mix: {count} planted instances, n log-uniform [200, 20000], k 2..64, "
                                   f"pop {{32, 64, 128}}, {args.batch_iters} iterations, gww 0.1, master seed 7 + rank",
                       "parallelism": f"replicas x{world}", "buckets": batch.describe()},
            "plain_solves_per_s": world * count / tp_all,
            "speedup_vs_plain": tp_all / tb_all,
            "engine": args.batch_engine,
            "latency_s": {"batched_p50": percentile(own, 0.5), "batched_p99": percentile(own, 0.99),
                          "plain_fifo_p50": percentile(done, 0.5), "plain_fifo_p99": percentile(done, 0.99),
                          "note": "all instances arrive at once; batched: each instance's completion in the run"},
            "speedup_bound_one_slot_per_sm": sum(t_plain) / packed,
            "bit_exact_vs_plain": bool(exact),
            "clocks": clock_info,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_serving(args, rank, world, local):
    """The serving stream (cuda_graph_clustering_b200.workloads.serving_requests, master seed 11 + rank):
    requests arrive by a Poisson process in real time and are submitted to a ccb_server as they arrive
    (graph generated on the device at admission); the server admits by its HBM budget and advances every
    admitted request one iteration per step.  Latency = completion - arrival.  The baseline is a plain FIFO:
    the same requests solved one at a time in arrival order (graph generation + ccb_solver_pbils + label
    copy, timed per request), its completion times computed from those service times and the arrivals.
    Every served result is checked equal to its plain result."""
    import torch

    import cuda_graph_clustering_b200 as ccb
    from cuda_graph_clustering_b200.workloads import serving_requests

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800))
    reqs = serving_requests(args.serve_count, args.serve_rate, master=11 + rank, max_n=args.serve_max_n,
                            population=64, iterations=50)

    def params(r):
        return ccb.PbilsParams(k=r.k, population=r.population, iterations=r.iterations,
                               early_stop=r.iterations, seed=r.seed)

    def submit(sv, r):
        if r.erdos_renyi:
            return sv.submit_generated(params(r), r.n, density=r.density, seed=r.graph_seed)
        return sv.submit_generated(params(r), r.n, planted=True, parts=r.parts, p_in=r.p_in, p_out=r.p_out,
                                   flip=r.flip, seed=r.graph_seed)

    def plain(r):
        if r.erdos_renyi:
            g = ccb.DeviceGraph.erdos_renyi(r.n, r.density, r.graph_seed)
        else:
            g = ccb.DeviceGraph.planted(r.n, r.parts, r.p_in, r.p_out, r.flip, r.graph_seed)[0]
        s_ = ccb.Solver(g, params(r))
        out = s_.pbils(params(r))
        s_.close()
        g.close()
        return out

    # warm-up: module loading and first-launch costs of every kernel family on a few small requests
    warm = [r for _, r in serving_requests(64, 1.0, master=1000 + rank, max_n=3000)][:max(args.warmup, 3)]
    sv = ccb.Server(hbm_budget_bytes=int(args.serve_budget_gb * 2**30))
    for r in warm:
        submit(sv, r)
        plain(r)
    sv.drain()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    clocks.start()
    finish = {}
    results = {}
    ids = {}
    nxt = 0
    peak_active = 0
    t0 = time.perf_counter()
    while len(finish) < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt][0] <= now:
            ids[submit(sv, reqs[nxt][1])] = nxt
            nxt += 1
        q, a, _ = sv.status()
        peak_active = max(peak_active, a)
        if q == 0 and a == 0:
            if nxt < len(reqs):
                time.sleep(max(0.0, reqs[nxt][0] - (time.perf_counter() - t0)))
            continue
        for i in sv.step():
            finish[ids[i]] = time.perf_counter() - t0
            results[ids[i]] = sv.result(i)
    t_serve = max(finish.values())
    clock_info = clocks.stop()
    sv.close()

    service = []
    exact = True
    for j, (_, r) in enumerate(reqs):
        t1 = time.perf_counter()
        w = plain(r)
        service.append(time.perf_counter() - t1)
        g = results[j]
        exact &= (w.objective == g.objective and w.iterations_done == g.iterations_done
                  and w.accepted_moves == g.accepted_moves and bool((w.labels == g.labels).all()))
    fifo = []
    free_at = 0.0
    for (arr, _), sdur in zip(reqs, service):
        free_at = max(free_at, arr) + sdur
        fifo.append(free_at)
    t_fifo = fifo[-1]
    (ts_all, tf_all), _ = combine_over_ranks(dist, [t_serve, t_fifo], [])
    if rank == 0:
        lat_s = [finish[j] - reqs[j][0] for j in range(len(reqs))]
        lat_f = [fifo[j] - reqs[j][0] for j in range(len(reqs))]
        count = len(reqs)
        line = {
            "metric": "serving solves/s", "value": world * count / ts_all, "unit": "solves/s", "n_gpus": world,
            "steps": 1, "warmup": len(warm), "ms_per_step": 1e3 * ts_all, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16/int32", "data": "synthetic",
            "config": {"workload": f"serving: {count} requests (first of the seeded stream, master seed 11 + rank), "
                                   f"Poisson {args.serve_rate}/s, ER or planted, n log-uniform [500, "
                                   f"{args.serve_max_n}], density [0.01, 0.5], k 2..32, pop 64, 50 iterations; "
                                   "graphs generated on the device at admission",
                       "parallelism": f"replicas x{world}",
                       "hbm_budget_bytes": int(args.serve_budget_gb * 2**30) or "80% of free"},
            "plain_fifo_solves_per_s": world * count / tf_all,
            "speedup_vs_plain_fifo": tf_all / ts_all,
            "latency_s": {"served_p50": percentile(sorted(lat_s), 0.5), "served_p99": percentile(sorted(lat_s), 0.99),
                          "plain_fifo_p50": percentile(sorted(lat_f), 0.5),
                          "plain_fifo_p99": percentile(sorted(lat_f), 0.99)},
            "peak_active": peak_active,
            "bit_exact_vs_plain": bool(exact),
            "clocks": clock_info,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_neighborhood(args, rank, world, local):
    """The Neighborhood configuration (NEIGHBORHOOD): one step = one NeighborhoodWithManyLocalSearchesCuda solve
    (all 4096 start partitions, each followed by a local search) on the device-resident graph; the solve without
    the local search (NeighborhoodCuda) is timed beside it.  Metric: accepted local-search moves per second.
    Every step's objective, moves and labels must equal tests/golden/neighborhood_reference.json (the oracle's
    and the reference's brute force, which agreed).  `e2e`: the one-call ABI from a pinned host bitset."""
    import hashlib

    import numpy as np
    import torch

    import cuda_graph_clustering_b200 as ccb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    c = NEIGHBORHOOD
    golden = json.load(open(os.path.join(REPO, "tests", "golden", "neighborhood_reference.json")))
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    dg, _ = ccb.DeviceGraph.planted(c["n"], c["parts"], c["p_in"], c["p_out"], c["flip"], c["graph_seed"],
                                    shuffle_split=c["shuffle_split"], stream=sh)
    graph = dg.download()
    params = ccb.PbilsParams(k=2, population=c["batch"])
    solver = ccb.Solver(dg, params)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def exact(r, key):
        w = golden[key]
        return (r.objective == w["objective"] and r.accepted_moves == w["accepted_moves"]
                and hashlib.sha256(np.asarray(r.labels, dtype="<i4").tobytes()).hexdigest() == w["labels_sha256"])

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        solver.neighborhood(params, True, stream=sh)
        solver.neighborhood(params, False, stream=sh)
    clocks = ClockSampler(local)
    timed = {}
    results = {}
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    for ls in (True, False):
        events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
        out = []
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                events[i][0].record(stream)
            out.append(solver.neighborhood(params, ls, stream=sh))
            events[i][1].record(stream)
        torch.cuda.synchronize()
        timed[ls] = sum(a.elapsed_time(b) for a, b in events)
        results[ls] = out
    barrier()
    clock_info = clocks.stop()
    bit_exact = all(exact(r, "local_search") for r in results[True]) and \
        all(exact(r, "plain") for r in results[False])

    solver.set_profiling(True)
    prof = solver.neighborhood(params, True, stream=sh)
    st = solver.stats()
    solver.set_profiling(False)
    descent_ms = st.descent_ms / max(st.descent_launches, 1)

    pinned = torch.empty(graph.bits.size, dtype=torch.int32, pin_memory=True)
    pinned.numpy().view(np.uint32)[:] = graph.bits.reshape(-1)
    g_pinned = ccb.Graph(graph.n, pinned.numpy().view(np.uint32).reshape(graph.bits.shape), graph.edges)
    ccb.SolveNeighborhoodWithManyLocalSearchesGpu(g_pinned, params)
    barrier()
    t0 = time.perf_counter()
    e2e_ok = True
    for _ in range(args.steps):
        e2e_ok &= exact(ccb.SolveNeighborhoodWithManyLocalSearchesGpu(g_pinned, params), "local_search")
    e2e_s = time.perf_counter() - t0
    moves = sum(r.accepted_moves for r in results[True])
    (t_ls, t_plain, t_e2e), (moves_all,) = combine_over_ranks(dist, [timed[True], timed[False], e2e_s], [moves])

    if rank == 0:
        n = c["n"]
        words = (n + 31) // 32
        deg = 2.0 * graph.edges / n
        moves_per_launch = prof.accepted_moves / max(st.descent_launches, 1)
        per_move = n * (2 * 2 + 1) + 4 * words + 8 * deg  # SURVEY 8(d) generic move bytes at k = 2, sG = 2
        modelled = moves_per_launch * per_move / (descent_ms * 1e-3) / 1e9
        peak, peak_kind = measured_peak_hbm()
        # the register descent (k = 2, 1024 threads x 4 vertices): issue roofline with the instructions per move
        # of its own ncu summary (profiles/k_descent_neighborhood.txt), the modelled bytes beside
        inst_per_move = profiled_value("k_descent_neighborhood", "warp_inst_per_move_per_block")
        sm_hz = (clock_info.get("sm_mhz") or 1965.0) * 1e6
        issue_peak = torch.cuda.get_device_properties(local).multi_processor_count * 4 * sm_hz / 1e9
        ach = (inst_per_move or 0.0) * moves_per_launch / (descent_ms * 1e-3) / 1e9
        nb_roofline = {"bound": "issue", "achieved": ach if inst_per_move else None, "peak": issue_peak,
                       "unit": "G warp-inst/s", "frac": ach / issue_peak if inst_per_move else None,
                       "traffic": profiled_traffic("k_descent_neighborhood"), "kernel": "k_descent_registers",
                       "avg_launch_ms": descent_ms,
                       "limiter": "instruction issue (72 % of active cycles, ALU pipe 82 % on the SMs in use); "
                                  "instructions per move from "
                                  "profiles/k_descent_neighborhood.txt",
                       "modelled_bytes": {"achieved_gbs": modelled, "hbm_peak_gbs": peak, "hbm_peak_kind": peak_kind,
                                          "frac_of_hbm": modelled / peak,
                                          "per_move": "n(2k+1) + 4 ceil(n/32) + 8 deg (SURVEY 8(d))"}}
        cpu = None
        if not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(REPO, "oracle"))
            from oracle import Reference
            if Reference.available():
                sample = 512
                t1 = time.perf_counter()
                _, ref_moves = Reference().neighborhood_range(graph.bits, True, 0, sample)
                dt = time.perf_counter() - t1
                cpu = {"value": ref_moves / dt, "unit": "moves/s", "cores": 1, "kind": "reference",
                       "sample": f"start vertices 0..{sample - 1} of {n} with the local search (the reference's "
                                 "sequential brute force, cuda/cc_verify_gpu.cu:21-35, on its own CPU State)",
                       "neighborhoods_per_s": sample / dt}
        line = {
            "metric": "Neighborhood LS moves/s", "value": moves_all / (t_ls * 1e-3), "unit": "moves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ls / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic",
            "config": {"workload": f"Neighborhood k=2: planted n={n} split 2048/2048 (seeded permutation, graph seed "
                                   f"{c['graph_seed']}), p_in {c['p_in']}, p_out {c['p_out']}, batch {c['batch']}, "
                                   "NeighborhoodWithManyLocalSearchesCuda (all start vertices)",
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                       "kernel_plan": solver.describe()},
            "neighborhoods_per_s": world * n * args.steps / (t_ls * 1e-3),
            "plain_neighborhood_solves_per_s": world * args.steps / (t_plain * 1e-3),
            "bit_exact": bool(bit_exact),
            "objective": results[True][0].objective,
            "e2e": {"value": moves_all / t_e2e, "unit": "moves/s", "h2d_bytes_per_step": int(graph.bits.nbytes),
                    "d2h_bytes_per_step": int(4 * n + 48), "bit_exact": bool(e2e_ok)},
            "roofline": nb_roofline,
            "kernel_ms_per_solve": {"descent": st.descent_ms, "rebuild": st.rebuild_ms, "record": st.record_ms,
                                    "other": st.other_ms},
            # per step pair: the solve with the local search, and the one without (no descent launches)
            "gpu_launches": int(args.steps * (st.descent_launches + 2 * (st.rebuild_launches + st.record_launches
                                                                         + st.other_launches))),
            "clocks": clock_info,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    if args.workload == "serving":
        run_serving(args, rank, world, local)
        return
    if args.workload == "neighborhood":
        run_neighborhood(args, rank, world, local)
        return

    import numpy as np
    import torch

    import cuda_graph_clustering_b200 as ccb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    cfg, objectives = WORKLOADS[args.workload]
    cfg = dict(cfg)
    seed = cfg["seed"] + rank
    if cfg["n"] > 20000:  # the device generator gives the same bits in milliseconds
        graph = ccb.DeviceGraph.erdos_renyi(cfg["n"], cfg["density"], cfg["graph_seed"]).download()
    else:
        graph = ccb.Graph.ErdosRenyi(cfg["n"], cfg["density"], cfg["graph_seed"])
    params = ccb.PbilsParams(k=cfg["k"], population=cfg["population"], tournament=cfg["tournament"],
                             perturbation=cfg["perturbation"], gww=cfg["gww"], iterations=cfg["iterations"],
                             early_stop=cfg["early_stop"], seed=seed)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    dg = ccb.DeviceGraph(graph, stream=sh)
    solver = ccb.Solver(dg, params)
    if args.rebuild != "auto":
        solver.set_rebuild(args.rebuild)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    expected = objectives.get(seed)

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident solves -------------------------------------------------------------
    for _ in range(args.warmup):
        r = solver.pbils(params, stream=sh)
    solver.set_profiling(False)
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    results = []
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            events[i][0].record(stream)
        results.append(solver.pbils(params, stream=sh, want_labels=False))
        events[i][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in events]
    total_ms = sum(step_ms)
    iters = sum(r.iterations_done for r in results)
    moves = sum(r.accepted_moves for r in results)
    bit_exact = all(r.objective == expected for r in results) if expected is not None else None

    # ---- per-kernel times (separate profiled pass: CUDA events around every launch) ----------
    solver.set_profiling(True)
    prof = solver.pbils(params, stream=sh, want_labels=False)
    st = solver.stats()
    rebuild_compare = None
    if "tensor cores" in solver.describe():
        # the same solve with the popcount rebuild: identical trajectory, the rebuild phase timed beside
        solver.set_rebuild("popcount")
        alt = solver.pbils(params, stream=sh, want_labels=False)
        st_pop = solver.stats()
        solver.set_rebuild(args.rebuild)
        n_, k_, pop_ = cfg["n"], cfg["k"], cfg["population"]
        ops = 2.0 * n_ * n_ * pop_ * k_ * st.rebuild_launches  # int8 MACs x 2 of every rebuild (initial included)
        rebuild_compare = {"tensor_ms_per_solve": st.rebuild_ms, "popcount_ms_per_solve": st_pop.rebuild_ms,
                           "launches": st.rebuild_launches, "same_objective": alt.objective == prof.objective,
                           "tensor_phase_tops": ops / (st.rebuild_ms * 1e-3) / 1e12,
                           "note": "rebuild phase = labels/masks/sizes + one-hot Z + tcgen05 contraction + f"}
    solver.set_profiling(False)
    descent_ms = st.descent_ms / max(st.descent_launches, 1)
    launches_per_solve = st.descent_launches + st.rebuild_launches + st.record_launches + st.other_launches

    # ---- end to end through the public one-call ABI ------------------------------------------
    pinned = torch.empty(graph.bits.size, dtype=torch.int32, pin_memory=True)
    pinned.numpy().view(np.uint32)[:] = graph.bits.reshape(-1)
    pbits = pinned.numpy().view(np.uint32).reshape(graph.bits.shape)
    g_pinned = ccb.Graph(graph.n, pbits, graph.edges)
    for _ in range(max(1, args.warmup // 2)):
        ccb.SolveGpu(g_pinned, params)
    barrier()
    t0 = time.perf_counter()
    e2e_ok = True
    e2e_results = []
    for _ in range(args.steps):
        r = ccb.SolveGpu(g_pinned, params)
        e2e_results.append(r)
        e2e_ok &= (expected is None or r.objective == expected)
    e2e_s = time.perf_counter() - t0
    recount_ok = None
    if expected is None:
        # size-independent check: the labels returned recount on the GPU to the reported objective, and the
        # e2e solves (same seed) give the device-resident solves' objective
        from cuda_graph_clustering_b200.cli import recount

        recount_ok = all(recount(graph, np.asarray(r.labels), cfg["k"]) == r.objective for r in e2e_results[:1])
        recount_ok &= all(r.objective == results[0].objective for r in e2e_results)
        bit_exact = recount_ok and all(r.objective == results[0].objective for r in results)

    # ---- max over ranks ------------------------------------------------------------------------
    (total_ms_all, e2e_all), (iters_all, moves_all) = combine_over_ranks(dist, [total_ms, e2e_s], [iters, moves])

    if rank == 0:
        n, k, pop = cfg["n"], cfg["k"], cfg["population"]
        words = (n + 31) // 32
        deg = 2.0 * graph.edges / n
        ld = (n + 31) // 32 * 32
        moves_per_launch = prof.accepted_moves / max(st.descent_launches, 1)
        # algorithmic bytes of one descent launch: per move n*(k*2 + 1) + 4*words + 4*2*deg (scan of the
        # state, the moved vertex's row, two G entries per neighbour), plus per slot the state copied in
        # (k*ld*2 + ld) and the labels written out (ld)
        per_move = n * (k * 2 + 1) + 4 * words + 8 * deg
        per_launch = moves_per_launch * per_move + pop * (k * ld * 2 + 2 * ld)
        if cfg["n"] > 32767 and k in (2, 3):
            # packed wide descent: per move the slot's words (4 or 8 bytes per vertex), the moved vertex's row
            # and the changed words of its neighbours; per slot the int32 G and labels read, labels written.
            # The degree-proportional forms read no full scan per move: the moved vertex's row and a read and
            # a write of each neighbour's word (their rescans, rare, are not counted).
            wb = 4 if k == 2 else 8
            per_move = wb * n + 4 * words + wb * deg
            if "degree-proportional" in solver.describe():
                per_move = 4 * words + 2 * wb * deg
            per_launch = moves_per_launch * per_move + pop * (k * ld * 4 + 2 * ld + wb * n)
        peak, peak_kind = measured_peak_hbm()
        achieved = per_launch / (descent_ms * 1e-3) / 1e9
        traffic = profiled_traffic(f"k_descent_{args.workload}")
        l2_peak, int8_peak = measured_peaks()
        modelled = {"achieved_gbs": achieved, "hbm_peak_gbs": peak, "hbm_peak_kind": peak_kind,
                    "frac_of_hbm": achieved / peak, "bytes_per_launch": per_launch,
                    "basis": "SURVEY 8(d) algorithmic bytes per accepted move (a modelled rate: the state is "
                             "read from registers, shared memory or L2)"}
        plan = solver.describe()
        if "registers" in plan and "incremental" not in plan:
            # the register descent: bound by the latency of its per-move chain, seen as issue utilisation
            inst_per_move = profiled_value("k_descent_plain", "warp_inst_per_move_per_block")
            sm_hz = (clock_info.get("sm_mhz") or 1965.0) * 1e6
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            issue_peak = sms * 4 * sm_hz / 1e9
            ach = (inst_per_move or 0.0) * moves_per_launch / (descent_ms * 1e-3) / 1e9
            roofline = {"bound": "issue", "achieved": ach, "peak": issue_peak, "unit": "G warp-inst/s",
                        "frac": ach / issue_peak, "traffic": traffic, "kernel": "k_descent_registers",
                        "avg_launch_ms": descent_ms,
                        "limiter": "latency of the per-move chain (row word, scan, warp minimum, block barrier); "
                                   "instructions per move from profiles/k_descent_plain.txt",
                        "peak_kind": "issue slots of all SMs (4 per SM per cycle) at the sampled SM clock",
                        "modelled_bytes": modelled}
        elif "L2" in plan and l2_peak:
            roofline = {"bound": "l2", "achieved": achieved, "peak": l2_peak, "unit": "GB/s",
                        "frac": achieved / l2_peak, "traffic": traffic, "kernel": "k_descent",
                        "avg_launch_ms": descent_ms, "peak_kind": "measured L2 copy (profiles/peaks_l2_hbm_int8.txt)",
                        "basis": modelled["basis"], "modelled_bytes": modelled}
        elif "degree-proportional" in plan and args.workload == "wide2" and \
                profiled_value("k_descent_wide2_sparse_n65536", "warp_inst_per_move_per_block"):
            # the W k = 2 descent (int16 state in shared memory): issue roofline with the instructions per move of
            # its own ncu summary, the modelled bytes beside
            inst_per_move = profiled_value("k_descent_wide2_sparse_n65536", "warp_inst_per_move_per_block")
            sm_hz = (clock_info.get("sm_mhz") or 1965.0) * 1e6
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            issue_peak = sms * 4 * sm_hz / 1e9
            ach = inst_per_move * moves_per_launch / (descent_ms * 1e-3) / 1e9
            roofline = {"bound": "issue", "achieved": ach, "peak": issue_peak, "unit": "G warp-inst/s",
                        "frac": ach / issue_peak, "traffic": traffic, "kernel": "k_descent_wide2_sparse",
                        "avg_launch_ms": descent_ms,
                        "limiter": "instruction issue under divergence; instructions per move from "
                                   "profiles/k_descent_wide2_sparse_n65536.txt",
                        "peak_kind": "issue slots of all SMs (4 per SM per cycle) at the sampled SM clock",
                        "ns_per_move_per_slot": descent_ms * 1e6 / max(moves_per_launch / pop, 1.0),
                        "modelled_bytes": modelled}
        elif "degree-proportional" in plan:
            # the sparse wide descents: per move one bitset row and the moved vertex's neighbours; the SMs holding
            # a slot issue on ~2/3 of their cycles with half the lanes idle (divergent neighbour loops), so
            # instruction issue, not bandwidth, sets the pace; the modelled bytes against HBM show how far from a
            # memory bound it runs
            roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": traffic, "peak_kind": peak_kind, "kernel": "k_descent_wide_sparse",
                        "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": descent_ms,
                        "limiter": "instruction issue under divergence (0.69 issue per active cycle, 16.8 of 32 "
                                   "lanes; profiles/k_descent_wide2_sparse_n65536.txt); the slot's state "
                                   + ("in shared memory" if " in shared memory," in plan else "in L2"),
                        "ns_per_move_per_slot": descent_ms * 1e6 / max(moves_per_launch / pop, 1.0)}
        else:
            roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": traffic, "peak_kind": peak_kind, "kernel": "k_descent",
                        "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": descent_ms}
        if rebuild_compare is not None and int8_peak:
            rebuild_compare["int8_peak_tops"] = int8_peak
            rebuild_compare["tensor_phase_frac_of_int8_peak"] = rebuild_compare["tensor_phase_tops"] / int8_peak
        value = iters_all / (total_ms_all * 1e-3)
        cpu = None
        have_ref = os.path.exists(os.path.join(REPO, "oracle", "_ref", "cc_cpu"))
        if cfg["n"] > 32767 and not args.no_cpu_baseline and have_ref:
            # one iteration at population 8 (its time includes the initial rebuild of the 8 slots), scaled to
            # the configuration's population 128: CPU time per iteration grows in proportion to the population
            small = dict(cfg, population=8)
            t, f, threads = reference_cpu_run(small, 1)
            cpu = {"value": 8.0 / (cfg["population"] * t), "unit": "iter/s", "cores": threads, "kind": "reference",
                   "sample": f"1 iteration at population 8 ({t:.1f} s, initial rebuild included), scaled by 8/128 "
                             "to population 128; --threads 0"}
        elif not args.no_cpu_baseline and have_ref:
            sample = 20 if args.workload == "plain" else 1
            t, f, threads = reference_cpu_run(cfg, sample)
            cpu = {"value": sample / t, "unit": "iter/s", "cores": threads, "kind": "reference",
                   "sample": f"{sample} of the {cfg['iterations']} iterations of the same instance and seed, "
                             "--threads 0"}
        ref_gpu = None
        if args.workload in ("plain", "gpucsv32k") and not args.no_cpu_baseline:
            got = reference_gpu_run(dict(cfg, seed=seed))
            if got is not None:
                t_ref, f_ref = got
                ref_gpu = {"value": cfg["iterations"] / t_ref, "unit": "iter/s", "objective": f_ref,
                           "same_objective": f_ref == results[0].objective,
                           "binary": "oracle/_ref/cc_gpu_ref: the reference's cuda/ sources built for sm_100a",
                           "timing": "its own solver time (PbilsResult.seconds, best of 3 runs; includes its "
                                     "per-call allocation and bitset upload)",
                           "ours_over_reference": value / (cfg["iterations"] / t_ref)}
        if args.workload in ("wide2", "wide3") and not args.no_cpu_baseline:
            # the reference's GPU design at W: a short run of both binaries through their one-call entry points
            # (5 iterations, same seed; both times include the per-call set-up and the 512 MiB bitset upload)
            short = 5
            got = reference_gpu_run(dict(cfg, seed=seed, iterations=short, early_stop=short), runs=1)
            if got is not None:
                t_ref, f_ref = got
                p_short = ccb.PbilsParams(k=cfg["k"], population=cfg["population"], tournament=cfg["tournament"],
                                          perturbation=cfg["perturbation"], gww=cfg["gww"], iterations=short,
                                          early_stop=short, seed=seed)
                t0 = time.perf_counter()
                r_short = ccb.SolveGpu(g_pinned, p_short)
                t_ours = time.perf_counter() - t0
                ref_gpu = {"value": short / t_ref, "unit": "iter/s", "objective": f_ref,
                           "same_objective": f_ref == r_short.objective, "iterations": short,
                           "ours_same_run": short / t_ours,
                           "binary": "oracle/_ref/cc_gpu_ref: the reference's cuda/ sources built for sm_100a",
                           "timing": "reference: its own solver time (PbilsResult.seconds, one run); ours: wall "
                                     "time of ccb_pbils_solve from the pinned host bitset; both include the "
                                     "per-call set-up and the bitset upload",
                           "ours_over_reference": t_ref / t_ours}
        line = {
            "metric": "PBILS iter/s", "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32" if n > 32767 else "int16",
            "data": "synthetic",
            "config": {"workload": workload_text(args.workload, cfg),
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                       "kernel_plan": solver.describe()},
            "ls_moves_per_s": moves_all / (total_ms_all * 1e-3),
            "bit_exact": bit_exact,
            "recount_ok": recount_ok,
            "objective": results[0].objective,
            "e2e": {"value": iters_all / e2e_all, "unit": "iter/s",
                    "h2d_bytes_per_step": int(graph.bits.nbytes), "d2h_bytes_per_step": int(4 * n + 48),
                    "bit_exact": e2e_ok},
            "roofline": roofline,
            "kernel_ms_per_solve": {"descent": st.descent_ms, "rebuild": st.rebuild_ms, "record": st.record_ms,
                                    "other": st.other_ms},
            "gpu_launches": int(launches_per_solve * args.steps),
            "clocks": clock_info,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "rebuild_tensor_vs_popcount": rebuild_compare,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
