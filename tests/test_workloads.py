"""The seeded benchmark workloads (batched mix, serving stream) are fixed by their master seeds: the bench's
inputs do not drift between runs or machines, and their parameters stay inside the stated ranges."""
from cuda_graph_clustering_b200.workloads import Draws, batched_mix, serving_requests, stream_seed


def test_streams_are_deterministic_and_distinct():
    a, b = Draws(7, 0xB47C4), Draws(7, 0xB47C4)
    assert [a.u64() for _ in range(5)] == [b.u64() for _ in range(5)]
    assert stream_seed(7, 1, 0) != stream_seed(7, 2, 0) != stream_seed(8, 1, 0)
    d = Draws(3, 1)
    assert all(0.0 <= d.unit() < 1.0 for _ in range(1000))
    assert all(0 <= d.below(5) < 5 for _ in range(1000))


def test_batched_mix_ranges_and_repeatability():
    mix = batched_mix(256, 7, iterations=100)
    assert mix == batched_mix(256, 7, iterations=100)
    assert mix != batched_mix(256, 8, iterations=100)
    assert len(mix) == 256
    for i in mix:
        assert 200 <= i.n <= 20000 and 2 <= i.parts <= 16 and 2 <= i.k <= 64
        assert 0.3 <= i.p_in <= 0.8 and 0.01 <= i.p_out <= 0.2 and 0.05 <= i.flip <= 0.2
        assert i.population in (32, 64, 128) and i.iterations == 100
    # the mix spans the whole k range and all three populations
    assert {i.population for i in mix} == {32, 64, 128}
    assert min(i.k for i in mix) <= 4 and max(i.k for i in mix) >= 60


def test_serving_stream_is_poisson_ordered_and_in_range():
    reqs = serving_requests(500, 100.0, master=11, max_n=50000, population=64, iterations=50)
    times = [t for t, _ in reqs]
    assert times == sorted(times) and times[0] > 0
    assert 3.0 < times[-1] < 7.0  # 500 arrivals at 100/s
    for _, r in reqs:
        assert 500 <= r.n <= 50000 and 2 <= r.k <= 32 and 0.01 <= r.density <= 0.5
        assert r.population == 64 and r.iterations == 50
    assert {r.erdos_renyi for _, r in reqs} == {True, False}
