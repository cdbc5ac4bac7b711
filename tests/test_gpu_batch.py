"""Device graph generation and the batched engine.

Generated graphs must equal the host generators bit for bit; every instance of a batch must give exactly
the result of its plain solve (and of the CPU oracle where that is quick)."""
import numpy as np
import pytest

from oracle import make_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 31, 32, 33, 100, 1000, 3001])
def test_device_erdos_renyi_matches_host(ccb, oracle, cuda_device, n):
    for density in (0.0, 0.33, 1.0):
        g = ccb.DeviceGraph.erdos_renyi(n, density, 7 + n).download()
        bits, edges = oracle.erdos_renyi(n, density, 7 + n)
        assert g.edges == edges and np.array_equal(g.bits, bits)


@pytest.mark.parametrize("n,parts,split", [(64, 2, True), (1000, 5, False), (2500, 2, True), (33, 3, False)])
def test_device_planted_matches_host(ccb, oracle, cuda_device, n, parts, split):
    dg, comm = ccb.DeviceGraph.planted(n, parts, 0.6, 0.1, 0.07, 11, shuffle_split=split)
    g = dg.download()
    bits, edges, comm_o = oracle.planted(n, parts, split, 0.6, 0.1, 0.07, 11)
    assert g.edges == edges and np.array_equal(g.bits, bits) and np.array_equal(comm, comm_o)


MIX = [
    # n, k, pop, gww, tournament, iterations, early_stop, perturbation, seed
    (60, 2, 8, 0.1, 5, 6, 6, 0.4, 1),
    (300, 5, 32, 0.25, 5, 10, 4, 0.4, 2),
    (1000, 3, 64, 0.1, 3, 8, 100, 0.3, 3),
    (1500, 8, 16, 0.0, 5, 5, 2, 0.4, 4),
    (4500, 4, 8, 0.1, 5, 2, 6, 0.4, 5),
    (700, 12, 32, 0.1, 5, 6, 6, 0.4, 6),
    (2500, 33, 8, 0.5, 5, 3, 6, 0.4, 7),
    (200, 64, 12, 0.1, 5, 4, 6, 0.4, 8),
    (5, 2, 3, 0.0, 2, 0, 6, 0.4, 9),
    (90, 1, 4, 0.1, 5, 3, 6, 0.4, 10),
]


def test_batch_matches_plain_and_oracle(ccb, oracle, cuda_device):
    batch = ccb.Batch()
    graphs, params, ids = [], [], []
    for i, (n, k, pop, gww, tour, iters, early, pert, seed) in enumerate(MIX):
        dg, _ = ccb.DeviceGraph.planted(n, max(2, k // 2), 0.5, 0.05, 0.1, 100 + i)
        p = ccb.PbilsParams(k=k, population=pop, gww=gww, tournament=tour, iterations=iters, early_stop=early,
                            perturbation=pert, seed=seed)
        graphs.append(dg)
        params.append(p)
        ids.append(batch.add(dg, p))
    batch.run()
    for i, (dg, p) in enumerate(zip(graphs, params)):
        got = batch.result(ids[i])
        host = dg.download()
        want = ccb.SolveGpu(host, p)
        assert (got.objective, got.iterations_done, got.accepted_moves, got.local_searches, got.clusters_used) == \
            (want.objective, want.iterations_done, want.accepted_moves, want.local_searches, want.clusters_used), i
        assert np.array_equal(got.labels, want.labels), i
        if host.n <= 1500:
            o = oracle.pbils(host.bits, host.edges, make_params(k=p.k, population=p.population, gww=p.gww,
                                                                tournament=p.tournament, iterations=p.iterations,
                                                                early_stop=p.early_stop,
                                                                perturbation=p.perturbation, seed=p.seed))
            assert o.objective == got.objective and np.array_equal(o.labels, got.labels), i
    # a second run of the same batch reproduces every result
    first = [batch.result(i).objective for i in ids]
    batch.run()
    assert [batch.result(i).objective for i in ids] == first


def test_lockstep_engine_matches_flow_engine(ccb, cuda_device):
    """The lock-step engine (one graph replay per iteration of all instances) and the flow engine (each instance
    on its own) give every instance the same result."""
    runs = []
    for engine in ("lockstep", "flow"):
        batch = ccb.Batch(engine=engine)
        ids = []
        for i, (n, k, pop, gww, tour, iters, early, pert, seed) in enumerate(MIX):
            dg, _ = ccb.DeviceGraph.planted(n, max(2, k // 2), 0.5, 0.05, 0.1, 400 + i)
            ids.append(batch.add(dg, ccb.PbilsParams(k=k, population=pop, gww=gww, tournament=tour, iterations=iters,
                                                     early_stop=early, perturbation=pert, seed=seed)))
        batch.run()
        runs.append([batch.result(i) for i in ids])
        batch.close()
    for a, b in zip(*runs):
        assert _results_equal(a, b)


def test_flow_engine_bounded_wait_ends_with_timeout(ccb, cuda_device):
    """Host-side fault injection: one instance's work is never published, so the other instances finish and then
    every block of its bucket finds nothing to claim; after the 1 s wait limit the kernel gives up (no trap, no
    endless spin) and the run reports CCB_ERR_TIMEOUT.  The device stays usable for the next batch."""
    from cuda_graph_clustering_b200._native import CCB_ERR_TIMEOUT, CcbError
    batch = ccb.Batch(engine="flow", wait_limit_sec=1.0)
    graphs = [ccb.DeviceGraph.planted(300 + 50 * i, 3, 0.5, 0.05, 0.1, 500 + i)[0] for i in range(4)]
    for g in graphs:
        batch.add(g, ccb.PbilsParams(k=4, population=16, iterations=5, early_stop=5, seed=2))
    batch.withhold(2)
    with pytest.raises(CcbError) as e:
        batch.run()
    assert e.value.status == CCB_ERR_TIMEOUT and "wait limit" in str(e.value)
    batch.close()
    again = ccb.Batch(engine="flow", wait_limit_sec=1.0)
    ids = [again.add(g, ccb.PbilsParams(k=4, population=16, iterations=5, early_stop=5, seed=2)) for g in graphs]
    again.run()
    for g, i in zip(graphs, ids):
        assert _results_equal(again.result(i), ccb.SolveGpu(g.download(), ccb.PbilsParams(
            k=4, population=16, iterations=5, early_stop=5, seed=2)))


def test_flow_engine_reports_per_instance_completion(ccb, cuda_device):
    """Under the flow engine a small instance finishes long before a large one: its own completion time is
    reported, not the run's."""
    batch = ccb.Batch(engine="flow")
    small = batch.add(ccb.DeviceGraph.planted(200, 2, 0.5, 0.05, 0.1, 601)[0],
                      ccb.PbilsParams(k=3, population=32, iterations=3, early_stop=3, seed=1))
    large = batch.add(ccb.DeviceGraph.planted(12000, 8, 0.5, 0.05, 0.1, 602)[0],
                      ccb.PbilsParams(k=20, population=64, iterations=20, early_stop=20, seed=1))
    batch.run()
    ts, tl = batch.result(small).seconds, batch.result(large).seconds
    assert 0 < ts < tl
    assert ts < 0.5 * tl


@pytest.mark.parametrize("table", [
    [dict(kind=-1, n_min=0, n_max=1 << 20, k_min=0, k_max=64, use_kind=2, threads=256, blocks_per_sm=0,
          max_slots=0)],
    [dict(kind=-1, n_min=0, n_max=1 << 20, k_min=0, k_max=64, use_kind=2, threads=512, blocks_per_sm=1,
          max_slots=3)],
    [dict(kind=-1, n_min=0, n_max=1 << 20, k_min=0, k_max=64, use_kind=-1, threads=0, blocks_per_sm=2,
          max_slots=0)],
])
def test_tuned_batch_matches_plain(ccb, cuda_device, table):
    """Every tuning choice (global-state kernel, threads per slot, resident blocks, slot cap) runs the same
    trajectories."""
    before = ccb.get_tuning()
    ccb.set_tuning(table)
    try:
        batch = ccb.Batch()
        runs = []
        extra = [(9000, 20, 8, 0.1, 5, 2, 6, 0.4, 11), (17000, 12, 6, 0.1, 5, 2, 6, 0.4, 12),
                 (6000, 40, 10, 0.1, 5, 2, 6, 0.4, 13)]
        for i, (n, k, pop, gww, tour, iters, early, pert, seed) in enumerate(MIX + extra):
            dg, _ = ccb.DeviceGraph.planted(n, max(2, k // 2), 0.5, 0.05, 0.1, 300 + i)
            p = ccb.PbilsParams(k=k, population=pop, gww=gww, tournament=tour, iterations=iters,
                                early_stop=early, perturbation=pert, seed=seed)
            runs.append((dg, p, batch.add(dg, p)))
        batch.run()
        for dg, p, i in runs:
            got = batch.result(i)
            want = ccb.SolveGpu(dg.download(), p)
            assert _results_equal(got, want), (i, batch.describe())
    finally:
        ccb.set_tuning(before)


def _results_equal(a, b):
    return (a.objective, a.iterations_done, a.accepted_moves, a.local_searches, a.clusters_used) == \
        (b.objective, b.iterations_done, b.accepted_moves, b.local_searches, b.clusters_used) and \
        np.array_equal(a.labels, b.labels)


def test_server_same_alone_and_in_the_mix(ccb, cuda_device):
    """Requests served together with others, admitted at different steps under a tight memory budget and
    a small active cap, give exactly the result of the same request served alone and of its plain solve."""
    reqs = []
    lanes = MIX + [(9000, 12, 4, 0.1, 5, 2, 6, 0.4, 21), (3000, 20, 8, 0.1, 5, 3, 6, 0.4, 22)]
    for i, (n, k, pop, gww, tour, iters, early, pert, seed) in enumerate(lanes):
        host, _ = ccb.Graph.Planted(n, max(2, k // 2), 0.5, 0.05, 0.1, 200 + i)
        p = ccb.PbilsParams(k=k, population=pop, gww=gww, tournament=tour, iterations=iters, early_stop=early,
                            perturbation=pert, seed=seed)
        reqs.append((host, p))
    alone = []
    for host, p in reqs:
        sv = ccb.Server()
        i = sv.submit(host, p)
        out = sv.drain()
        alone.append(out[i])
        sv.close()
    sv = ccb.Server(hbm_budget_bytes=3 << 20, max_active=4)
    ids = [sv.submit(host, p) for host, p in reqs]
    # device-generated requests beside the host ones: one batched, one beyond the narrow limit (stepped on its own stream)
    gp = ccb.PbilsParams(k=6, population=16, iterations=5, early_stop=3, seed=12)
    gid = sv.submit_generated(gp, 900, planted=True, parts=3, p_in=0.6, p_out=0.1, flip=0.05, seed=77)
    wp = ccb.PbilsParams(k=5, population=4, iterations=2, early_stop=3, seed=13)
    wid = sv.submit_generated(wp, 34000, density=0.004, seed=78)
    seen_active = 0
    out = {}
    while True:
        for i in sv.step():
            out[i] = sv.result(i)
        q, a, b = sv.status()
        seen_active = max(seen_active, a)
        assert a <= 4
        if q == 0 and a == 0:
            break
    assert seen_active > 1
    for j, (host, p) in enumerate(reqs):
        want = ccb.SolveGpu(host, p)
        assert _results_equal(alone[j], want), j
        assert _results_equal(out[ids[j]], want), j
    dg, _ = ccb.DeviceGraph.planted(900, 3, 0.6, 0.1, 0.05, 77)
    assert _results_equal(out[gid], ccb.SolveGpu(dg.download(), gp))
    wg = ccb.DeviceGraph.erdos_renyi(34000, 0.004, 78)
    assert _results_equal(out[wid], ccb.SolveGpu(wg.download(), wp))
    sv.close()


def test_server_request_that_cannot_be_admitted_fails_alone(ccb, cuda_device):
    """A request whose buffers exceed the device memory fails at admission without allocating; its result
    carries the error and the requests around it are served as usual."""
    host, _ = ccb.Graph.Planted(1000, 3, 0.5, 0.05, 0.1, 31)
    small = ccb.PbilsParams(k=6, population=8, iterations=3, seed=4)
    sv = ccb.Server()
    bad = sv.submit(host, ccb.PbilsParams(k=64, population=5_000_000, iterations=1))
    good = sv.submit(host, small)
    results, errors = {}, {}
    while len(results) + len(errors) < 2:
        for i in sv.step():
            try:
                results[i] = sv.result(i)
            except ccb.CcbError as e:
                errors[i] = e
    assert set(errors) == {bad} and "device memory" in str(errors[bad])
    assert _results_equal(results[good], ccb.SolveGpu(host, small))
    sv.close()


def test_server_cancel_queued_and_admitted(ccb, cuda_device):
    """Cancelling a queued request removes it; cancelling an admitted one stops it before its lane's next
    iteration; both report CCB_ERR_CANCELLED, and the request served after them is unaffected."""
    host, _ = ccb.Graph.Planted(800, 4, 0.5, 0.05, 0.1, 41)
    ps = [ccb.PbilsParams(k=5, population=8, iterations=30, early_stop=30, seed=s) for s in (1, 2, 3)]
    sv = ccb.Server(max_active=1)
    ids = [sv.submit(host, p) for p in ps]
    sv.step()  # admits the first request and runs one of its iterations
    assert sv.cancel(ids[2]) and sv.cancel(ids[0]) and not sv.cancel(123456)
    results, errors = {}, {}
    while not (ids[0] in errors and ids[1] in results):
        for i in sv.step():
            try:
                results[i] = sv.result(i)
            except ccb.CcbError as e:
                errors[i] = e
    assert errors[ids[0]].status == ccb._native.CCB_ERR_CANCELLED
    with pytest.raises(ccb.CcbError) as queued:
        sv.result(ids[2])
    assert queued.value.status == ccb._native.CCB_ERR_CANCELLED
    assert _results_equal(results[ids[1]], ccb.SolveGpu(host, ps[1]))
    sv.close()


def test_server_steps_wide_requests_and_cancels_one(ccb, cuda_device):
    """Requests beyond the narrow limit are stepped by the server loop, a chunk of iterations at a time on their
    own streams, beside a batched lane: each finishes with its plain solve's result, and one cancelled while its
    chunk runs reports CCB_ERR_CANCELLED without disturbing the others."""
    sv = ccb.Server()
    wp = ccb.PbilsParams(k=3, population=8, iterations=12, early_stop=12, seed=5)
    a = sv.submit_generated(wp, 36000, density=0.003, seed=90)
    b = sv.submit_generated(wp, 40000, density=0.003, seed=91)
    np_ = ccb.PbilsParams(k=6, population=16, iterations=6, early_stop=6, seed=6)
    c = sv.submit_generated(np_, 1200, planted=True, parts=3, p_in=0.6, p_out=0.1, flip=0.05, seed=92)
    sv.step()  # all three admitted: two wide chunks and one lane iteration in flight
    assert sv.cancel(b)
    results, errors = {}, {}
    while len(results) + len(errors) < 3:
        for i in sv.step():
            try:
                results[i] = sv.result(i)
            except ccb.CcbError as e:
                errors[i] = e
    assert errors[b].status == ccb._native.CCB_ERR_CANCELLED
    assert _results_equal(results[a], ccb.SolveGpu(ccb.DeviceGraph.erdos_renyi(36000, 0.003, 90).download(), wp))
    dg, _ = ccb.DeviceGraph.planted(1200, 3, 0.6, 0.1, 0.05, 92)
    assert _results_equal(results[c], ccb.SolveGpu(dg.download(), np_))
    sv.close()
