"""GPU parity: the sm_100a kernels (through the C ABI) against the CPU oracle and the golden fixtures.

Every comparison is exact: objective, labels (tie-breaking), iterations done, accepted moves, local
searches and clusters used, as the reference's own GPU test compares them (cuda/cc_verify_gpu.cu:37-54).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import make_params
from tests.golden_graphs import graph_from_mask

pytestmark = pytest.mark.gpu

KERNELS = {"auto": 0, "global": 1, "shared": 2, "wide": 3}


def _graph(ccb, bits, edges):
    return ccb.Graph(bits.shape[0], bits, edges)


def _same(got, want, what=""):
    assert got.objective == want.objective, what
    assert got.iterations_done == want.iterations_done, what
    assert got.accepted_moves == want.accepted_moves, what
    assert got.local_searches == want.local_searches, what
    assert got.clusters_used == want.clusters_used, what
    assert np.array_equal(np.asarray(got.labels), np.asarray(want.labels)), what


def _params(ccb, **kw):
    return ccb.PbilsParams(**kw)


CASES = [
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
    (513, 0.05, 15, 6, 40, 5, 6, 6, 0.4, 0.1, 15),
    (1000, 0.33, 7, 3, 128, 5, 4, 1000, 0.4, 0.0, 6),
    (2100, 0.4, 16, 4, 20, 5, 2, 6, 0.4, 0.1, 16),
]


@pytest.mark.parametrize("case", CASES, ids=[f"n{c[0]}k{c[3]}p{c[4]}" for c in CASES])
@pytest.mark.parametrize("kernel", list(KERNELS))
def test_pbils_matches_oracle(ccb, oracle, cuda_device, case, kernel):
    n, density, gseed, k, pop, tour, iters, early, pert, gww, seed = case
    bits, edges = oracle.erdos_renyi(n, density, gseed)
    want = oracle.pbils(bits, edges, make_params(k=k, population=pop, tournament=tour, iterations=iters,
                                                 early_stop=early, perturbation=pert, gww=gww, seed=seed))
    got = ccb.SolveGpu(_graph(ccb, bits, edges),
                       _params(ccb, k=k, population=pop, tournament=tour, iterations=iters, early_stop=early,
                               perturbation=pert, gww=gww, seed=seed, ls_kernel=KERNELS[kernel]))
    _same(got, want, f"{case} {kernel}")


def test_reference_pbils_runs(ccb, oracle, reference_runs, cuda_device):
    for case in reference_runs["pbils"]:
        bits, edges = oracle.erdos_renyi(case["n"], case["density"], case["graph_seed"])
        for kernel in KERNELS.values():
            got = ccb.SolveGpu(_graph(ccb, bits, edges), _params(
                ccb, k=case["k"], population=case["population"], tournament=case["tournament"],
                iterations=case["iterations"], early_stop=case["early_stop"], perturbation=case["perturbation"],
                gww=case["gww"], seed=case["seed"], ls_kernel=kernel))
            assert (got.objective, got.iterations_done, got.clusters_used, got.local_searches,
                    got.accepted_moves) == (case["objective"], case["iterations_done"], case["clusters_used"],
                                            case["local_searches"], case["accepted_moves"]), (case["n"], kernel)
            assert got.labels.tolist() == case["labels"]


def test_iterations_zero_is_initial_record(ccb, oracle, cuda_device):
    bits, edges = oracle.erdos_renyi(300, 0.4, 5)
    for k in (1, 2, 5, 64):
        want = oracle.pbils(bits, edges, make_params(k=k, population=17, iterations=0, seed=9))
        got = ccb.SolveGpu(_graph(ccb, bits, edges), _params(ccb, k=k, population=17, iterations=0, seed=9))
        _same(got, want, f"k={k}")


# docs/data/gpu.csv rows (protocol of docs/gpu_sweep.sh:13-15), up to n = 8000
def test_published_gpu_csv(ccb, oracle, published, cuda_device):
    rows = [r for r in published["gpu_csv"] if r["n"] <= 8000 and r["pop"] <= 1024]
    assert len(rows) >= 60
    graphs = {}
    for r in rows:
        if r["n"] not in graphs:
            bits, edges = oracle.erdos_renyi(r["n"], 0.33, 7)
            graphs[r["n"]] = _graph(ccb, bits, edges)
        got = ccb.SolveGpu(graphs[r["n"]], _params(ccb, k=r["k"], population=r["pop"], iterations=20,
                                                  early_stop=1000, gww=0.0, seed=r["seed"]))
        assert got.objective == r["f"], f"gpu.csv:{r['line']}"
        assert got.iterations_done == 20


# docs/data/gww_stop.csv (default --iters 100 --early-stop 6): f and iteration count per seed
def test_published_gww_stop(ccb, oracle, published, cuda_device):
    rows = [r for r in published["gww_stop_csv"] if r["n"] <= 2000]
    assert len(rows) >= 100
    graphs = {}
    for r in rows:
        key = (r["n"], r["graph_seed"])
        if key not in graphs:
            bits, edges = oracle.erdos_renyi(r["n"], 0.33, r["graph_seed"])
            graphs[key] = _graph(ccb, bits, edges)
        got = ccb.SolveGpu(graphs[key], _params(ccb, k=r["k"], population=r["pop"], gww=r["gww"], seed=r["seed"]))
        assert (got.objective, got.iterations_done) == (r["f"], r["iters"]), f"gww_stop.csv:{r['line']}"


# docs/data/gww.csv: record at checkpoint iterations of 1000-iteration runs (no early stop)
def test_published_gww_long_runs(ccb, oracle, published, cuda_device):
    runs = [r for r in published["gww_csv"] if r["graph_seed"] == 7 and r["seed"] in (2, 3)]
    assert runs
    bits, edges = oracle.erdos_renyi(1000, 0.33, 7)
    g = _graph(ccb, bits, edges)
    for r in runs:
        for it, record in r["checkpoints"]:
            if it not in (1, 10, 100, r["iters"]):
                continue
            got = ccb.SolveGpu(g, _params(ccb, k=r["k"], population=r["pop"], gww=r["gww"], seed=r["seed"],
                                          iterations=it, early_stop=r["iters"]))
            assert got.objective == record, (r["first_line"], it)


# The plain configuration: ER(1000, 0.5, graph seed 1), k 5, pop 128, gww 0.1, seed 1.
def test_plain_config(ccb, oracle, cuda_device):
    bits, edges = oracle.erdos_renyi(1000, 0.5, 1)
    g = _graph(ccb, bits, edges)
    got = ccb.SolveGpu(g, _params(ccb, k=5, population=128, iterations=100, early_stop=100, seed=1))
    assert (got.objective, got.iterations_done) == (234911, 100)
    want = oracle.pbils(bits, edges, make_params(k=5, population=128, iterations=100, early_stop=100, seed=1))
    _same(got, want)
    got6 = ccb.SolveGpu(g, _params(ccb, k=5, population=128, iterations=100, seed=1))
    assert (got6.objective, got6.iterations_done) == (234924, 52)


def test_neighborhood_exhaustive_small(ccb, reference_runs, cuda_device):
    for case in reference_runs["neighborhood"]:
        if "mask" not in case:
            continue
        bits = graph_from_mask(case["n"], case["mask"])
        g = ccb.Graph(case["n"], bits)
        for key, fn in (("plain", ccb.SolveNeighborhoodGpu), ("ls", ccb.SolveNeighborhoodWithManyLocalSearchesGpu)):
            got = fn(g, _params(ccb, population=3))
            want = case[key]
            assert got.objective == want["objective"] and got.labels.tolist() == want["labels"], case
            assert got.accepted_moves == want["accepted_moves"] and got.clusters_used == want["clusters_used"]
            assert got.local_searches == (case["n"] if key == "ls" else 0)


def test_neighborhood_boundaries(ccb, oracle, reference_runs, cuda_device):
    for case in reference_runs["neighborhood"]:
        if "mask" in case:
            continue
        bits, edges = oracle.erdos_renyi(case["n"], case["density"], case["graph_seed"])
        g = _graph(ccb, bits, edges)
        runs = [(17, k) for k in KERNELS.values()] + [(1, 0), (case["n"] + 3, 0)]
        for batch, kernel in runs:
            for key, fn in (("plain", ccb.SolveNeighborhoodGpu),
                            ("ls", ccb.SolveNeighborhoodWithManyLocalSearchesGpu)):
                got = fn(g, _params(ccb, population=batch, ls_kernel=kernel))
                want = case[key]
                what = (case["n"], case["density"], batch, kernel, key)
                assert got.objective == want["objective"], what
                assert got.labels.tolist() == want["labels"], what
                assert got.accepted_moves == want["accepted_moves"], what
                assert got.clusters_used == want["clusters_used"], what


def test_neighborhood_planted_partial_batch(ccb, oracle, cuda_device):
    bits, edges, _ = oracle.planted(1024, 2, True, 0.6, 0.1, 0.0, 5)
    g = _graph(ccb, bits, edges)
    for ls in (False, True):
        want = oracle.neighborhood(bits, edges, ls)
        fn = ccb.SolveNeighborhoodWithManyLocalSearchesGpu if ls else ccb.SolveNeighborhoodGpu
        for batch in (128, 100):
            got = fn(g, _params(ccb, population=batch))
            _same(got, want, (ls, batch))


@pytest.mark.parametrize("k", [2, 3])
def test_wide_path_beyond_narrow_limit(ccb, oracle, cuda_device, k):
    n = 33000
    bits, edges = oracle.erdos_renyi(n, 0.01, 21)
    p = dict(k=k, population=6, iterations=2, early_stop=10, seed=3)
    want = oracle.pbils(bits, edges, make_params(**p))
    got = ccb.SolveGpu(_graph(ccb, bits, edges), _params(ccb, **p))
    _same(got, want)
    assert oracle.objective_bitwise(bits, got.labels) == got.objective


@pytest.mark.parametrize("n,k,density", [(40000, 12, 0.02), (50000, 30, 0.01), (65536, 2, 0.005),
                                         (65536, 3, 0.005), (70000, 2, 0.002), (70000, 3, 0.002),
                                         (34000, 2, 0.3), (34000, 3, 0.3), (33000, 3, 0.05)])
def test_wide_auto_matches_generic_wide(ccb, oracle, cuda_device, n, k, density):
    """Beyond the narrow limit the auto plan runs the packed descents for k = 2, 3 (one word per vertex; for
    k = 2 on a sparse graph the degree-proportional form) and the cached-key descent on uint16 counters with
    64-bit move keys for larger k (up to n = 65536); the forced generic wide kernel (int32 G, full scan) must
    give the same run."""
    g = ccb.DeviceGraph.erdos_renyi(n, density, 5 + k).download()
    p = dict(k=k, population=4, iterations=2, early_stop=10, seed=k)
    auto = ccb.SolveGpu(g, _params(ccb, **p))
    wide = ccb.SolveGpu(g, _params(ccb, ls_kernel=KERNELS["wide"], **p))
    _same(auto, wide)
    assert oracle.objective_bitwise(g.bits, auto.labels) == auto.objective


def test_solver_reuse_and_devicegraph(ccb, oracle, cuda_device):
    bits, edges = oracle.erdos_renyi(400, 0.3, 2)
    dg = ccb.DeviceGraph(_graph(ccb, bits, edges))
    s = ccb.Solver(dg, _params(ccb, k=4, population=24))
    for seed in (1, 2, 3):
        want = oracle.pbils(bits, edges, make_params(k=4, population=24, iterations=8, seed=seed))
        got = s.pbils(_params(ccb, k=4, population=24, iterations=8, seed=seed))
        _same(got, want, seed)
    with pytest.raises(RuntimeError):
        s.pbils(_params(ccb, k=3, population=24))


def test_shared_kernel_rejects_oversized_state(ccb, oracle, cuda_device):
    bits, edges = oracle.erdos_renyi(20000, 0.01, 2)
    with pytest.raises(RuntimeError) as e:
        ccb.SolveGpu(_graph(ccb, bits, edges), _params(ccb, k=16, population=2, iterations=1, ls_kernel=2))
    assert "bytes of shared memory, device allows" in str(e.value)


# 4096 < n: the streamed K <= 8 descent, state in shared memory (n * 16 B fits) and in L2 (it does not);
# k > 8: the incremental descent with cached keys in registers (n <= 16384; counters in shared memory or L2)
# and with everything in global memory (n > 16384)
@pytest.mark.parametrize("n,k,density", [(4500, 2, 0.3), (5000, 8, 0.2), (9000, 3, 0.1), (13000, 6, 0.05),
                                         (20000, 5, 0.02), (1500, 12, 0.3), (3000, 40, 0.1), (6000, 20, 0.05),
                                         (2500, 64, 0.5), (17000, 10, 0.01)])
def test_streamed_descent_matches_oracle(ccb, oracle, cuda_device, n, k, density):
    bits, edges = oracle.erdos_renyi(n, density, n + k)
    p = dict(k=k, population=4, iterations=2, early_stop=10, gww=0.25, seed=5)
    want = oracle.pbils(bits, edges, make_params(**p))
    got = ccb.SolveGpu(_graph(ccb, bits, edges), _params(ccb, **p))
    _same(got, want, (n, k))


def test_solvers_sharing_a_kernel_keep_their_shared_memory(ccb, oracle, cuda_device):
    # n = 1000 and n = 600 at k = 5 use the same descent instance (256 threads x 4 vertices, bitset in shared
    # memory) with different shared-memory sizes; creating the smaller one last must not break the larger.
    big_bits, big_e = oracle.erdos_renyi(1000, 0.4, 3)
    small_bits, small_e = oracle.erdos_renyi(600, 0.4, 4)
    p = ccb.PbilsParams(k=5, population=8, iterations=2)
    big = ccb.Solver(ccb.DeviceGraph(_graph(ccb, big_bits, big_e)), p)
    small = ccb.Solver(ccb.DeviceGraph(_graph(ccb, small_bits, small_e)), p)
    assert big.describe().split(",")[1:3] == small.describe().split(",")[1:3]
    want = oracle.pbils(big_bits, big_e, make_params(k=5, population=8, iterations=2))
    _same(big.pbils(p), want)
    _same(small.pbils(p), oracle.pbils(small_bits, small_e, make_params(k=5, population=8, iterations=2)))


def test_one_call_cache_reuses_buffers_exactly(ccb, oracle, cuda_device):
    """Repeated one-call solves of the same shape reuse the cached device buffers (a new bitset each time);
    every result equals the oracle's, also after the cache is released and for a different graph."""
    p = dict(k=4, population=16, iterations=5, seed=2)
    for graph_seed in (3, 4, 3):
        bits, edges = oracle.erdos_renyi(500, 0.3, graph_seed)
        want = oracle.pbils(bits, edges, make_params(**p))
        _same(ccb.SolveGpu(_graph(ccb, bits, edges), _params(ccb, **p)), want, graph_seed)
    ccb.lib().ccb_release_cache()
    bits, edges = oracle.erdos_renyi(500, 0.3, 4)
    _same(ccb.SolveGpu(_graph(ccb, bits, edges), _params(ccb, **p)),
          oracle.pbils(bits, edges, make_params(**p)), "after release")


_WIDE_GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                        "wide_reference.json")))


@pytest.mark.parametrize("run", _WIDE_GOLDEN, ids=lambda r: f"n{r['n']}_k{r['k']}_p{r['density']}")
def test_matches_the_reference_binary_at_large_sizes(ccb, cuda_device, run):
    """At n = 65536 (the wide configuration's size, at p = 0.005 and at its own p = 0.02) and at n = 32000,
    k = 8 (the narrow limit's large configuration) the GPU run equals the reference's own CPU solver
    (tests/golden/make_wide_golden.py ran oracle/_ref/cc_cpu): objective, iterations, clusters used and the
    labels' SHA-256."""
    g = ccb.DeviceGraph.erdos_renyi(run["n"], run["density"], run["graph_seed"]).download()
    got = ccb.SolveGpu(g, _params(ccb, k=run["k"], population=run["population"], iterations=run["iterations"],
                                  seed=run["seed"]))
    assert (got.objective, got.iterations_done, got.clusters_used) == \
        (run["objective"], run["iterations_done"], run["clusters_used"])
    labels = np.asarray(got.labels, dtype="<i4")
    assert hashlib.sha256(labels.tobytes()).hexdigest() == run["labels_sha256"]
