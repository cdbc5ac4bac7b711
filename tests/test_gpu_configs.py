"""GPU parity at the benchmark configurations themselves (all through the C ABI, all exact).

* Neighborhood: the planted n = 4096 graph (2048/2048, p_in 0.6, p_out 0.1) with batches of 128 (32 full
  batches) and 100 (a partial last batch), both algorithms, against tests/golden/neighborhood_reference.json
  (the oracle's and the reference's own brute force, cuda/cc_verify_gpu.cu:21-35, which agreed).
* The narrow limit: the published docs/data/gpu.csv rows with n = 12000 ... 32000 (k = 3, pop 128 and 1024),
  the streamed small-k descent at the sizes of the n = 32000 configuration.
* The batched mix at its own 100 iterations: a seeded subset that spans every bucket kind, each instance equal
  to its plain solve and, where the CPU oracle is quick, to the oracle.
* The device-side time limit (Progress::Next's time rule, include/cc_pbils.hpp:69-78): a run cut short stops
  between iterations with a consistent record, equal to the run of exactly that many iterations.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import make_params

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sha(labels):
    return hashlib.sha256(np.asarray(labels, dtype="<i4").tobytes()).hexdigest()


def _same(a, b, what=""):
    assert (a.objective, a.iterations_done, a.accepted_moves, a.local_searches, a.clusters_used) == \
        (b.objective, b.iterations_done, b.accepted_moves, b.local_searches, b.clusters_used), what
    assert np.array_equal(np.asarray(a.labels), np.asarray(b.labels)), what


def test_neighborhood_configuration_n4096(ccb, cuda_device):
    golden = json.load(open(os.path.join(GOLDEN, "neighborhood_reference.json")))
    dg, _ = ccb.DeviceGraph.planted(golden["n"], golden["parts"], golden["p_in"], golden["p_out"], golden["flip"],
                                    golden["graph_seed"], shuffle_split=golden["shuffle_split"])
    g = dg.download()
    assert g.edges == golden["edges"]
    for key, fn in (("plain", ccb.SolveNeighborhoodGpu), ("local_search", ccb.SolveNeighborhoodWithManyLocalSearchesGpu)):
        want = golden[key]
        for batch in (128, 100):  # 4096 / 100: 40 full batches and a last one of 96
            got = fn(g, ccb.PbilsParams(k=2, population=batch))
            what = (key, batch)
            assert (got.objective, got.accepted_moves, got.clusters_used, got.local_searches) == \
                (want["objective"], want["accepted_moves"], want["clusters_used"], want["local_searches"]), what
            assert _sha(got.labels) == want["labels_sha256"], what
            if key == "plain":  # the chosen start vertex's closed neighbourhood is the label-0 side
                v = want["tie_break_vertex"]
                row = np.unpackbits(g.bits[v].view(np.uint8), bitorder="little")[: g.n].astype(bool)
                row[v] = True
                assert np.array_equal(np.asarray(got.labels) == 0, row), what


def test_published_gpu_csv_narrow_limit(ccb, published, cuda_device):
    """docs/data/gpu.csv rows with n > 8000 (ER(n, 0.33, graph seed 7), 20 iterations, gww 0, seed 5 + run):
    the streamed descent up to the narrow limit n = 32000."""
    rows = [r for r in published["gpu_csv"] if r["n"] > 8000]
    assert {r["n"] for r in rows} == {12000, 16000, 24000, 32000}
    graphs = {}
    for r in rows:
        if r["n"] not in graphs:
            graphs[r["n"]] = ccb.DeviceGraph.erdos_renyi(r["n"], 0.33, 7)
        s = ccb.Solver(graphs[r["n"]], ccb.PbilsParams(k=r["k"], population=r["pop"]))
        got = s.pbils(ccb.PbilsParams(k=r["k"], population=r["pop"], iterations=20, early_stop=1000, gww=0.0,
                                      seed=r["seed"]))
        s.close()
        assert (got.objective, got.iterations_done) == (r["f"], 20), f"gpu.csv:{r['line']}"


def _mix_subset(ccb, iterations):
    """Instances of the batched mix (master seed 7) covering each descent family of the plan: registers
    (k <= 8, n <= 4096), streamed (k <= 8, n > 4096), incremental with cached keys (k > 8, n <= 16384) and
    incremental in global memory (k > 8, n > 16384); the two cheapest of each."""
    from cuda_graph_clustering_b200.workloads import batched_mix
    mix = batched_mix(256, 7, iterations)
    kinds = {}
    for i, inst in enumerate(mix):
        kind = ("registers" if inst.n <= 4096 else "stream") if inst.k <= 8 else \
            ("incremental-regs" if inst.n <= 16384 else "incremental")
        kinds.setdefault(kind, []).append((inst.n * inst.population * min(inst.k, 16), i))
    assert set(kinds) == {"registers", "stream", "incremental-regs", "incremental"}
    return [mix[i] for kind in sorted(kinds) for _, i in sorted(kinds[kind])[:2]]


@pytest.mark.parametrize("engine", ["lockstep", "flow"])
def test_batched_mix_at_100_iterations(ccb, oracle, cuda_device, engine):
    subset = _mix_subset(ccb, 100)
    batch = ccb.Batch(engine=engine)
    runs = []
    for inst in subset:
        dg, _ = ccb.DeviceGraph.planted(inst.n, inst.parts, inst.p_in, inst.p_out, inst.flip, inst.graph_seed)
        p = ccb.PbilsParams(k=inst.k, population=inst.population, iterations=inst.iterations,
                            early_stop=inst.iterations, gww=0.1, seed=inst.seed)
        runs.append((inst, dg, p, batch.add(dg, p)))
    batch.run()
    for inst, dg, p, i in runs:
        got = batch.result(i)
        host = dg.download()
        _same(got, ccb.SolveGpu(host, p), (inst.n, inst.k, inst.population))
        assert got.iterations_done == 100
        if inst.n * inst.population <= 1000 * 64:
            o = oracle.pbils(host.bits, host.edges, make_params(k=p.k, population=p.population, iterations=100,
                                                                early_stop=100, gww=0.1, seed=p.seed))
            assert o.objective == got.objective and np.array_equal(o.labels, got.labels), inst.n


def test_time_limit_stops_between_iterations(ccb, oracle, cuda_device):
    """A 0.25 s limit on a run of 100000 iterations: the device's record kernel stops it after the iteration
    in which the limit passed (Progress::Next), so the result is that of exactly iterations_done iterations
    and its objective is the recount of its labels."""
    bits, edges = oracle.erdos_renyi(3000, 0.3, 4)
    g = ccb.Graph(3000, bits, edges)
    p = dict(k=6, population=64, early_stop=100000, seed=3)
    cut = ccb.SolveGpu(g, ccb.PbilsParams(iterations=100000, time_limit_sec=0.25, **p))
    assert 0 < cut.iterations_done < 100000
    assert cut.seconds < 30
    assert oracle.objective_bitwise(bits, cut.labels) == cut.objective
    exact = ccb.SolveGpu(g, ccb.PbilsParams(iterations=cut.iterations_done, **p))
    _same(cut, exact)
