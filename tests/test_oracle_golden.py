"""Pins the CPU oracle (oracle/cc_oracle.c) to the reference's published results and known answers.

Golden rows come from the reference's own result tables (docs/data/*.csv, extracted into
tests/golden/published.json by tests/golden/make_golden.py) and from runs of the reference's own
CPU code (tests/golden/reference_runs.json).  Only cases the oracle finishes in seconds run here;
the GPU tests cover the rest of each table.
"""
import numpy as np
import pytest

from oracle import make_params


def _gnp(oracle, n, density, seed):
    return oracle.erdos_renyi(n, density, seed)


# docs/data/gpu.csv: --density 0.33 --graph-seed 7 --iters 20 --early-stop 1000 --gww 0, seed 5 + run
@pytest.mark.parametrize("n,k,pop", [(1000, 3, 128), (2000, 2, 128)])
def test_gpu_csv_rows(oracle, published, n, k, pop):
    rows = [r for r in published["gpu_csv"] if r["n"] == n and r["k"] == k and r["pop"] == pop]
    assert rows, "no published row"
    bits, edges = _gnp(oracle, n, 0.33, 7)
    for r in rows[:2]:
        p = make_params(k=k, population=pop, iterations=20, early_stop=1000, gww=0.0, seed=r["seed"])
        sol = oracle.pbils(bits, edges, p)
        assert sol.objective == r["f"] == r["cpu_f"], f"gpu.csv:{r['line']}"
        assert sol.iterations_done == 20


# docs/data/cpu.csv 'ours' rows: 5 iterations, gww 0, seed 5 + rep
def test_cpu_csv_rows(oracle, published):
    rows = [r for r in published["cpu_csv"] if r["n"] in (500, 1000) and r["threads"] == 16]
    assert len(rows) >= 10
    cache = {}
    for r in rows[:12]:
        if r["n"] not in cache:
            cache[r["n"]] = _gnp(oracle, r["n"], 0.33, 7)
        bits, edges = cache[r["n"]]
        p = make_params(k=r["k"], population=r["pop"], iterations=5, early_stop=1000, gww=0.0, seed=r["seed"])
        assert oracle.pbils(bits, edges, p).objective == r["f"], f"cpu.csv:{r['line']}"


# docs/data/gww_stop.csv: default --iters 100 --early-stop 6, --gww share, seeds 2..9
def test_gww_stop_rows(oracle, published):
    rows = [r for r in published["gww_stop_csv"] if r["n"] == 1000 and r["graph_seed"] == 7]
    assert rows
    bits, edges = _gnp(oracle, 1000, 0.33, 7)
    picked = [r for r in rows if r["seed"] == 2][:4]
    for r in picked:
        p = make_params(k=r["k"], population=r["pop"], gww=r["gww"], seed=r["seed"])
        sol = oracle.pbils(bits, edges, p)
        assert (sol.objective, sol.iterations_done) == (r["f"], r["iters"]), f"gww_stop.csv:{r['line']}"


def test_reference_pbils_runs(oracle, reference_runs):
    for case in reference_runs["pbils"]:
        bits, edges = _gnp(oracle, case["n"], case["density"], case["graph_seed"])
        assert edges == case["edges"]
        p = make_params(k=case["k"], population=case["population"], tournament=case["tournament"],
                        iterations=case["iterations"], early_stop=case["early_stop"],
                        perturbation=case["perturbation"], gww=case["gww"], seed=case["seed"])
        sol = oracle.pbils(bits, edges, p, threads=3)
        got = (sol.objective, sol.iterations_done, sol.clusters_used, sol.local_searches, sol.accepted_moves)
        want = (case["objective"], case["iterations_done"], case["clusters_used"], case["local_searches"],
                case["accepted_moves"])
        assert got == want, case
        assert sol.labels.tolist() == case["labels"]


def test_reference_neighborhood_runs(oracle, reference_runs):
    from tests.golden_graphs import graph_from_mask
    for case in reference_runs["neighborhood"]:
        if "mask" in case:
            bits = graph_from_mask(case["n"], case["mask"])
            edges = int(sum(int(x).bit_count() for x in bits.ravel())) // 2
        else:
            bits, edges = _gnp(oracle, case["n"], case["density"], case["graph_seed"])
        for key, ls in (("plain", False), ("ls", True)):
            sol = oracle.neighborhood(bits, edges, ls, threads=2)
            want = case[key]
            assert sol.objective == want["objective"]
            assert sol.labels.tolist() == want["labels"]
            assert sol.accepted_moves == want["accepted_moves"]
            assert sol.clusters_used == want["clusters_used"]


# Known answers of the reference's CPU tests (src/cc_verify.cpp:131-178, :236-257, :377-399)
def test_known_optima(oracle):
    # complete graph -> one cluster, f = 0
    for n in (2, 6, 33):
        bits, edges = _gnp(oracle, n, 1.0, 1)
        f, labels, _ = oracle.local_search(bits, edges, 3, np.arange(n) % 3)
        assert f == 0 and len(set(labels.tolist())) == 1
    # edgeless K4 with k = 2: all together f = 6, optimum 2
    bits = np.zeros((4, 1), np.uint32)
    assert oracle.rebuild(bits, 0, 2, np.zeros(4, np.int32))[0] == 6
    assert oracle.local_search(bits, 0, 2, np.zeros(4, np.int32))[0] == 2
    # two disjoint triangles split for free at k = 2
    bits = np.zeros((6, 1), np.uint32)
    for a, b in ((0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5)):
        bits[a, 0] |= 1 << b
        bits[b, 0] |= 1 << a
    assert oracle.local_search(bits, 6, 2, np.array([0, 1, 0, 1, 0, 1], np.int32))[0] == 0
    # n = 1
    assert oracle.rebuild(np.zeros((1, 1), np.uint32), 0, 2, np.zeros(1, np.int32))[0] == 0


def test_edgeless_balanced_split(oracle):
    for n in (6, 9, 12):
        for k in (2, 3, 4):
            bits = np.zeros((n, 1), np.uint32)
            rng = np.random.default_rng(n * 31 + k)
            f, _, _ = oracle.local_search(bits, 0, k, rng.integers(0, k, n).astype(np.int32))
            base, rem = divmod(n, k)
            want = sum((base + (c < rem)) * (base + (c < rem) - 1) // 2 for c in range(k))
            assert f == want


def test_objective_forms_agree(oracle):
    rng = np.random.default_rng(31337)
    for n in (1, 2, 31, 32, 33, 63, 64, 65, 200):
        for density in (0.0, 0.3, 1.0):
            bits, edges = _gnp(oracle, n, density, int(rng.integers(1 << 30)))
            for k in (1, 2, 3, 7):
                labels = rng.integers(0, k, n).astype(np.int32)
                direct = oracle.objective_direct(bits, labels)
                assert oracle.objective_bitwise(bits, labels) == direct
                assert oracle.rebuild(bits, edges, k, labels)[0] == direct


def test_gww_slot_order(oracle):
    assert oracle.rank_slots([5, 3, 5, 1, 3]).tolist() == [3, 1, 4, 0, 2]
    assert oracle.lib.orc_winner_copies(0.1, 128) == 12
    assert oracle.lib.orc_winner_copies(0.5, 7) == 3


def test_thread_count_independent(oracle):
    bits, edges = _gnp(oracle, 150, 0.4, 99)
    p = make_params(k=3, population=24, iterations=15, early_stop=15, gww=0.25)
    one = oracle.pbils(bits, edges, p, threads=1)
    four = oracle.pbils(bits, edges, p, threads=4)
    assert (one.objective, one.iterations_done) == (four.objective, four.iterations_done)
    assert np.array_equal(one.labels, four.labels)
