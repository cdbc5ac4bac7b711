"""CPU-side checks of the C ABI library: it loads, exports every declared symbol, its host generators
emit the oracle's bits, and parameter errors carry the reference's messages (these are raised before
any CUDA call, so no device is needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for header in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not header.endswith(".h"):
            continue
        text = open(os.path.join(REPO, "include", header)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(ccb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(ccb):
    lib = C.CDLL(ccb._native.library_path())
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_defaults(ccb):
    p = ccb.CcbParams()
    ccb.lib().ccb_params_init(C.byref(p))
    assert (p.k, p.population, p.tournament, p.iterations, p.early_stop) == (2, 128, 5, 100, 6)
    assert (p.perturbation, p.gww, p.seed, p.ls_kernel) == (0.4, 0.1, 1, 0)
    d = ccb.PbilsParams()
    assert (d.k, d.population, d.tournament, d.iterations, d.early_stop, d.perturbation, d.gww, d.seed) == \
        (p.k, p.population, p.tournament, p.iterations, p.early_stop, p.perturbation, p.gww, p.seed)


@pytest.mark.parametrize("n,density,seed", [(0, 0.5, 1), (1, 0.3, 2), (33, 0.5, 3), (257, 0.1, 4), (700, 0.9, 5)])
def test_erdos_renyi_matches_oracle(ccb, oracle, n, density, seed):
    g = ccb.Graph.ErdosRenyi(n, density, seed)
    bits, edges = oracle.erdos_renyi(n, density, seed)
    assert g.edges == edges and np.array_equal(g.bits, bits)


@pytest.mark.parametrize("n,parts,split,pin,pout,flip,seed", [
    (64, 2, True, 0.6, 0.1, 0.0, 1), (4096 // 8, 2, True, 0.6, 0.1, 0.0, 9), (300, 5, False, 0.7, 0.05, 0.1, 7),
    (1, 3, False, 0.5, 0.5, 0.5, 2), (0, 2, True, 0.5, 0.5, 0.0, 3)])
def test_planted_matches_oracle(ccb, oracle, n, parts, split, pin, pout, flip, seed):
    g, comm = ccb.Graph.Planted(n, parts, pin, pout, flip, seed, shuffle_split=split)
    bits, edges, comm_o = oracle.planted(n, parts, split, pin, pout, flip, seed)
    assert g.edges == edges and np.array_equal(g.bits, bits) and np.array_equal(comm, comm_o)
    if split and n:
        assert (comm == 0).sum() == n // 2


@pytest.mark.parametrize("params,message", [
    (dict(k=0), "k must be >= 1"),
    (dict(population=0), "population must be >= 1"),
    (dict(gww=0.6), "gww must be in [0, 0.5]"),
    (dict(gww=-0.1), "gww must be in [0, 0.5]"),
    (dict(k=65), "k exceeds kMaxClusters (64); raise it in cc_gpu.hpp and rebuild"),
])
def test_pbils_rejects_bad_params(ccb, params, message):
    g = ccb.Graph.ErdosRenyi(10, 0.5, 1)
    with pytest.raises(RuntimeError) as e:
        ccb.SolveGpu(g, ccb.PbilsParams(**params))
    assert str(e.value) == message
    assert e.value.status == 1


@pytest.mark.parametrize("n,params,message", [
    (5, dict(k=3), "Neighborhood algorithms require k = 2"),
    (5, dict(population=0), "population must be >= 1"),
    (0, dict(), "Neighborhood requires 1 <= n <= 1048576"),
])
def test_neighborhood_rejects_bad_input(ccb, n, params, message):
    g = ccb.Graph.ErdosRenyi(n, 0.5, 1)
    for fn in (ccb.SolveNeighborhoodGpu, ccb.SolveNeighborhoodWithManyLocalSearchesGpu):
        with pytest.raises(RuntimeError) as e:
            fn(g, ccb.PbilsParams(**params))
        assert str(e.value) == message


def test_empty_graph_pbils_needs_no_device(ccb):
    # The reference records every offer on an empty graph (its label vector stays empty), so the stall
    # never grows and all iterations run; with early_stop 0 the first iteration stops.
    r = ccb.SolveGpu(ccb.Graph(0), ccb.PbilsParams(iterations=7, population=3))
    assert (r.objective, r.iterations_done, r.local_searches, r.clusters_used) == (0, 7, 21, 0)
    r = ccb.SolveGpu(ccb.Graph(0), ccb.PbilsParams(iterations=7, early_stop=0))
    assert r.iterations_done == 1


def test_tuning_table_roundtrip(ccb):
    entries = [dict(kind=3, n_min=8193, n_max=16384, k_min=9, k_max=64, use_kind=2, threads=256, blocks_per_sm=0,
                    max_slots=0),
               dict(kind=1, n_min=4097, n_max=32767, k_min=2, k_max=8, use_kind=-1, threads=0, blocks_per_sm=1,
                    max_slots=148)]
    before = ccb.get_tuning()
    try:
        ccb.set_tuning(entries)
        assert ccb.get_tuning() == entries
        ccb.set_tuning([])
        assert ccb.get_tuning() == []
        with pytest.raises(ccb.CcbError):
            ccb.check(ccb.lib().ccb_tuning_set(None, 1))
    finally:
        ccb.set_tuning(before)


def test_committed_tuning_table_is_well_formed(ccb):
    path = ccb.TUNING_PATH
    if not os.path.exists(path):
        pytest.skip("no tuning table committed")
    import json
    table = json.load(open(path))
    for e in table["entries"]:
        assert set(e) == set(ccb.TUNING_FIELDS)
        assert e["kind"] in (-1, 0, 1, 2, 3) and e["use_kind"] in (-1, 2)
        assert e["n_min"] <= e["n_max"] and e["k_min"] <= e["k_max"]
        assert e["use_kind"] == -1 or e["threads"] in (256, 512, 1024)
