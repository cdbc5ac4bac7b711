"""The oracle restatement against the reference's own CPU code (oracle/_ref/libccref.so), case by case."""
import numpy as np
import pytest

from oracle import make_params


def test_stream_primitives(oracle, reference):
    rng = np.random.default_rng(5)
    for _ in range(200):
        seed, stream, step = (int(x) for x in rng.integers(0, 2**63, 3, dtype=np.uint64))
        assert oracle.lib.orc_stream_seed(seed, stream, step) == reference.lib.ref_stream_seed(seed, stream, step)
        base = oracle.lib.orc_stream_seed(seed, 0xA11CE, 0)
        for k in (1, 2, 5, 64):
            idx = int(rng.integers(0, 2**40))
            assert oracle.lib.orc_initial_label(base, idx, k) == reference.lib.ref_initial_label(base, idx, k)
            it = int(rng.integers(0, 1000))
            lab = int(rng.integers(0, k))
            for p in (0.0, 0.4, 1.0):
                assert (oracle.lib.orc_perturbed_label(base, idx, it, lab, k, p)
                        == reference.lib.ref_perturbed_label(base, idx, it, lab, k, p))
        f = rng.integers(0, 5, 37).astype(np.int64)
        for t in (1, 2, 5, 9):
            assert (oracle.lib.orc_tournament(base, 3, 7, f, 37, t)
                    == reference.lib.ref_tournament(base, 3, 7, f, 37, t))


def test_erdos_renyi_bits(oracle, reference):
    for n, p, s in [(0, 0.5, 1), (1, 0.5, 1), (31, 0.2, 3), (32, 0.5, 4), (33, 0.9, 5), (500, 0.33, 7)]:
        a, ea = oracle.erdos_renyi(n, p, s)
        b, eb = reference.erdos_renyi(n, p, s)
        assert ea == eb and np.array_equal(a, b)


def test_rebuild_and_local_search(oracle, reference):
    rng = np.random.default_rng(11)
    for n in (1, 5, 31, 64, 97, 200):
        for k in (1, 2, 3, 7, 64):
            bits, edges = oracle.erdos_renyi(n, float(rng.uniform(0.1, 0.9)), int(rng.integers(1 << 30)))
            labels = rng.integers(0, k, n).astype(np.int32)
            fo, go, so = oracle.rebuild(bits, edges, k, labels)
            fr, gr, sr = reference.rebuild(bits, k, labels)
            assert fo == fr and np.array_equal(go, gr) and np.array_equal(so, sr)
            lo = oracle.local_search(bits, edges, k, labels)
            lr = reference.local_search(bits, k, labels)
            assert lo[0] == lr[0] and lo[2] == lr[2] and np.array_equal(lo[1], lr[1])


def test_rank_slots(oracle, reference):
    rng = np.random.default_rng(3)
    for pop in (1, 2, 7, 128, 513):
        f = rng.integers(0, 6, pop).astype(np.int64)
        order = np.zeros(pop, np.int32)
        reference.lib.ref_rank_slots(f, pop, order)
        assert np.array_equal(oracle.rank_slots(f), order)


@pytest.mark.parametrize("case", [
    dict(n=60, density=0.5, k=4, population=12, tournament=3, iterations=9, early_stop=3, perturbation=0.3,
         gww=0.25, seed=42),
    dict(n=130, density=0.2, k=9, population=20, tournament=5, iterations=6, early_stop=6, perturbation=0.6,
         gww=0.1, seed=7),
    dict(n=90, density=0.8, k=2, population=33, tournament=1, iterations=8, early_stop=100, perturbation=0.0,
         gww=0.5, seed=3),
])
def test_pbils_matches_reference(oracle, reference, case):
    bits, edges = oracle.erdos_renyi(case["n"], case["density"], 1234)
    p = make_params(**{k: v for k, v in case.items() if k not in ("n", "density")})
    a = oracle.pbils(bits, edges, p, threads=3)
    b = reference.pbils(bits, p, threads=2)
    assert (a.objective, a.iterations_done, a.clusters_used, a.local_searches, a.accepted_moves) == \
        (b.objective, b.iterations_done, b.clusters_used, b.local_searches, b.accepted_moves)
    assert np.array_equal(a.labels, b.labels)
