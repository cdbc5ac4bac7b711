"""Golden runs of the reference's own CPU solver at the wide size (n = 65536), for the wide-path parity test.

    python tests/golden/make_wide_golden.py

Runs oracle/_ref/cc_cpu (the reference's CPU binary, built from its sources by oracle/Makefile) on G(65536, p)
for k = 2 and k = 3 with a small population, and records the objective, the iteration count and a SHA-256 of
the labels (int32, little-endian) in tests/golden/wide_reference.json.  The GPU test regenerates the same graph
on the device and must reproduce all three.
"""
import hashlib
import json
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
CC_CPU = os.path.join(REPO, "oracle", "_ref", "cc_cpu")
RUNS = [dict(n=65536, density=0.005, graph_seed=3, k=2, population=4, iterations=2, seed=9),
        dict(n=65536, density=0.005, graph_seed=3, k=3, population=4, iterations=2, seed=10)]


def main():
    out = []
    for r in RUNS:
        with tempfile.TemporaryDirectory() as tmp:
            labels_path = os.path.join(tmp, "labels.txt")
            cmd = [CC_CPU, "--n", str(r["n"]), "--density", str(r["density"]), "--graph-seed", str(r["graph_seed"]),
                   "--k", str(r["k"]), "--pop", str(r["population"]), "--iters", str(r["iterations"]),
                   "--seed", str(r["seed"]), "--threads", "0", "--no-verify", "--labels-out", labels_path]
            text = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
            labels = np.array(open(labels_path).read().split(), dtype=np.int32)
        m = re.search(r"run 0\s+f=(\d+)\s+clusters=(\d+)\s+iters=(\d+)", text)
        out.append(dict(r, objective=int(m.group(1)), clusters_used=int(m.group(2)), iterations_done=int(m.group(3)),
                        labels_sha256=hashlib.sha256(labels.astype("<i4").tobytes()).hexdigest()))
        print(out[-1])
    with open(os.path.join(HERE, "wide_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
