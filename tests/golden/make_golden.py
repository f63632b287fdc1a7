"""Regenerate tests/golden/golden.json with the CPU oracle.

Run from the repository root after building the oracle:

    python tests/golden/make_golden.py [--reference-data DIR]

Records, for every synthetic workload the tests and the benchmark use, the
result size, the LIE iteration counts, the per-iteration trace and the
order-sensitive digest of the sorted result (the same digest the engine's
gdl_relation_digest computes).  With --reference-data (the reference
project's data/ directory), it also records, for the edge lists whose
same-generation sizes the reference publishes (README.md:80-103, computed
there by test/cuDF/sg.py), the file's SHA-256 and the oracle's answer, so
the CPU tests can pin the oracle against those published numbers.  The
dataset files themselves are not copied.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "gdlog-multinode_b200"))

import programs as P  # noqa: E402
import workloads as W  # noqa: E402
from gdlog_b200 import Engine  # noqa: E402

# Same-generation sizes published by the reference (README.md:83-103 and
# test/cuDF/sg.json), keyed by data file.  Iterations there are cuDF's loop
# count, not the engine's.
PUBLISHED_SG = {
    "data_5.txt": 4,
    "data_7035.txt": 285431,
    "data_21693.txt": 23519,
    "data_23874.txt": 608090,
    "data_121544.txt": 647999,
    "data_119666.txt": 245221,
}


def run(prog, *args):
    eng = Engine("oracle")
    t0 = time.time()
    r = prog(eng, *args)
    out = {
        "sizes": {k: v.size() for k, v in r.relations.items()},
        "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
        "iterations": r.iterations,
        "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
        "oracle_seconds": round(time.time() - t0, 3),
    }
    eng.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-data", default=None)
    ap.add_argument("--skip-large", action="store_true")
    args = ap.parse_args()
    g = {"workloads": {}, "published_sg": {}}
    W_ = g["workloads"]
    W_["tc_grid_64x64"] = run(P.tc, W.grid_edges(64, 64))
    W_["tc_grid_16x16"] = run(P.tc, W.grid_edges(16, 16))
    for seed in (1, 2, 3):
        W_[f"tc_dag_L12_W10_s{seed}"] = run(P.tc, W.layered_dag(12, 10, seed))
        W_[f"sg_rmat_s8_600_s{seed}"] = run(P.sg, W.rmat_edges(8, 600, seed=seed))
        W_[f"cspa_v120_s{seed}"] = run(P.cspa, *W.cspa_facts(120, 240, 90, seed=seed))
    W_["cspa_v300_s3"] = run(P.cspa, *W.cspa_facts(300, 600, 225, seed=3))
    W_["sg_rmat_s10_4096_s14"] = run(P.sg, W.rmat_edges(10, 4096, seed=14))
    if not args.skip_large:
        W_["sg_rmat_s14_40000_s14"] = run(P.sg, W.rmat_edges(14, 40000, seed=14))
    if args.reference_data:
        for name, size in PUBLISHED_SG.items():
            path = os.path.join(args.reference_data, name)
            if not os.path.exists(path):
                continue
            sha = hashlib.sha256(open(path, "rb").read()).hexdigest()
            res = run(P.sg, W.read_tsv(path))
            g["published_sg"][name] = {
                "sha256": sha,
                "published_size": size,
                "oracle": {"size": res["sizes"]["sg"], "iterations": res["iterations"],
                           "digest": res["digests"]["sg"]},
            }
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
