"""The cc_gpu command line mirror: edge-list loading and argument handling on the CPU; a full run on the GPU
checked against the oracle, with the reference's result-JSON keys and labels file."""
import json
import os

import pytest

from oracle import make_params


def test_edge_list_ranks_ids_and_skips_comments(tmp_path):
    from cuda_graph_clustering_b200.cli import load_edge_list

    p = tmp_path / "e.txt"
    p.write_text("# comment\n% other\nsrc,dst\n10 20\n20 30 extra\n30,10\n5 5\n100\t10\n")
    g = load_edge_list(str(p))
    # ids 5, 10, 20, 30, 100 -> vertices 0..4; the self-loop on 5 keeps its vertex but adds no edge
    assert g.n == 5 and g.edges == 4
    pairs = {(1, 2), (2, 3), (3, 1), (4, 1)}
    for i in range(5):
        for j in range(5):
            assert g.IsJoined(i, j) == ((i, j) in pairs or (j, i) in pairs)


def test_edge_list_without_edges_is_an_error(tmp_path, capsys):
    from cuda_graph_clustering_b200.cli import main

    p = tmp_path / "empty.txt"
    p.write_text("# nothing\n")
    assert main(["--edges", str(p)]) == 1
    assert "error: no edges in" in capsys.readouterr().out


def test_parser_defaults_match_reference_params():
    from cuda_graph_clustering_b200.cli import parser

    a = parser().parse_args([])
    assert (a.k, a.pop, a.tournament, a.iters, a.early_stop, a.perturb, a.gww, a.seed) == \
        (2, 128, 5, 100, 6, 0.4, 0.1, 1)
    assert (a.n, a.density, a.graph_seed, a.runs) == (500, 0.5, 1, 1)  # cli::Options (include/cc_cli.hpp:30-51)
    assert a.algorithm == "pbils" and a.ls_kernel == "auto" and a.verify


@pytest.mark.gpu
def test_cli_run_writes_reference_json(tmp_path, oracle, cuda_device, capsys):
    from cuda_graph_clustering_b200.cli import main

    out, labels = tmp_path / "r.json", tmp_path / "l.txt"
    rc = main(["--n", "300", "--density", "0.3", "--graph-seed", "4", "--k", "4", "--pop", "16", "--iters", "6",
               "--runs", "2", "--out", str(out), "--labels-out", str(labels)])
    assert rc == 0
    text = capsys.readouterr().out
    assert "verified" in text and "objective    min=" in text
    r = json.loads(out.read_text())
    keys = ["algorithm", "backend", "size", "edges", "density", "k", "population", "gww", "runs",
            "objective function value", "objective average", "objective max", "computation time seconds",
            "computation time average", "clusters used", "clustering vector"]
    assert list(r) == keys
    bits, edges = oracle.erdos_renyi(300, 0.3, 4)
    runs = [oracle.pbils(bits, edges, make_params(k=4, population=16, iterations=6, seed=s)) for s in (1, 2)]
    best = min(runs, key=lambda x: x.objective)
    assert r["objective function value"] == best.objective and r["objective max"] == max(x.objective for x in runs)
    assert r["clustering vector"] == [int(x) for x in best.labels]
    assert [int(x) for x in labels.read_text().split()] == [int(x) for x in best.labels]


CC_GPU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cuda_graph_clustering_b200",
                      "cc_gpu")


def _cc_gpu(*args):
    import subprocess

    return subprocess.run([CC_GPU, *args], capture_output=True, text=True, timeout=300)


@pytest.mark.skipif(not os.path.exists(CC_GPU), reason="drop-in cc_gpu not built (needs the reference sources)")
def test_drop_in_cc_gpu_rejects_bad_parameters_like_the_reference():
    """The reference's own command line linked with libccb: parameter errors come back as the reference's
    messages and exit code before any device work."""
    r = _cc_gpu("--n", "10", "--k", "65")
    assert r.returncode == 1 and "error: k exceeds kMaxClusters (64)" in r.stdout
    r = _cc_gpu("--algorithm", "NeighborhoodCuda", "--n", "10", "--k", "3")
    assert r.returncode == 1 and "error: Neighborhood algorithms require k = 2" in r.stdout


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(CC_GPU), reason="drop-in cc_gpu not built (needs the reference sources)")
def test_drop_in_cc_gpu_solves_like_the_oracle(tmp_path, oracle, cuda_device):
    out = tmp_path / "r.json"
    r = _cc_gpu("--n", "300", "--density", "0.3", "--graph-seed", "4", "--k", "4", "--pop", "16", "--iters", "6",
                "--out", str(out))
    assert r.returncode == 0, r.stdout + r.stderr
    got = json.loads(out.read_text())
    bits, edges = oracle.erdos_renyi(300, 0.3, 4)
    want = oracle.pbils(bits, edges, make_params(k=4, population=16, iterations=6, seed=1))
    assert got["objective function value"] == want.objective
    assert got["clustering vector"] == [int(x) for x in want.labels]
    assert got["backend"] == "gpu"


REF_CPU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "cc_cpu")


@pytest.mark.skipif(not os.path.exists(REF_CPU), reason="reference CPU binary not built")
def test_result_json_matches_the_reference_writer(tmp_path):
    """write_result_json emits the reference's WriteResultJson text: the same lines in the same order with the
    same number formatting, except the backend name and the CPU-only threads line."""
    import subprocess
    from types import SimpleNamespace

    import numpy as np

    import cuda_graph_clustering_b200 as ccb
    from cuda_graph_clustering_b200.cli import parser, write_result_json

    ref_json = tmp_path / "ref.json"
    flags = ["--n", "120", "--density", "0.3", "--graph-seed", "5", "--k", "3", "--pop", "8", "--iters", "4",
             "--runs", "2"]
    subprocess.run([REF_CPU, *flags, "--out", str(ref_json)], check=True, capture_output=True, timeout=120)
    ref = json.loads(ref_json.read_text())
    graph = ccb.Graph.ErdosRenyi(120, 0.3, 5)
    best = SimpleNamespace(objective=ref["objective function value"], seconds=ref["computation time seconds"],
                           clusters_used=ref["clusters used"], labels=np.array(ref["clustering vector"]))
    ours = tmp_path / "ours.json"
    write_result_json(str(ours), graph, parser().parse_args(flags), best, ref["objective average"],
                      ref["objective max"], ref["computation time average"])
    keep = lambda text: [l for l in text.splitlines() if '"backend"' not in l and '"threads"' not in l]
    assert keep(ours.read_text()) == keep(ref_json.read_text())
