"""Record the answers of the points-to analysis (test/cspa.cu:100-379) on
inputs too large for the list oracle, computed by the bit-matrix oracle
(oracle/oracle_bitset.cpp, test infrastructure), into
tests/golden/cspa_large.json.

The list oracle materialises every join candidate; on the 20,000-variable
input (40,000 assign and 15,000 dereference pairs, source bounded Zipf(1.1),
target uniform, seed 3) that is about 13.7 T candidates.  The bit-matrix
oracle evaluates the same loop (src/lie.cu:26-274) with joins as boolean
matrix products and finishes it in about a minute on 8 host cores.  It is
pinned beside this fixture against the list oracle and the reference CUDA
build's own answers (tests/test_oracle_bitset.py).

Usage, from the repository root (no GPU needed):

    python tests/golden/make_cspa_large.py [--only NAME[,NAME...]]
"""
from __future__ import annotations

import argparse
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

OUT = os.path.join(HERE, "cspa_large.json")

# name -> inputs; cspa_c3 is the 20,000-variable configuration.
WORKLOADS = {
    "cspa_v2000_s3": lambda: W.cspa_facts(2000, 4000, 1500, seed=3),
    "cspa_v6000_s3": lambda: W.cspa_facts(6000, 12000, 4500, seed=3),
    "cspa_c3": lambda: W.cspa_facts(),
}


def run(name: str) -> dict:
    assign, deref = WORKLOADS[name]()
    with Engine("oracle_bitset") as e:
        t0 = time.perf_counter()
        r = P.cspa(e, assign, deref)
        secs = time.perf_counter() - t0
        return {
            "inputs": {"assign_rows": int(len(assign)), "dereference_rows": int(len(deref))},
            "sizes": {k: v.size() for k, v in r.relations.items()},
            "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
            "iterations": dict(r.iterations),
            "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
            "oracle": "oracle_bitset",
            "oracle_threads": e.threads,
            "oracle_seconds": round(secs, 2),
        }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=OUT)
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    names = a.only.split(",") if a.only else list(WORKLOADS)
    res = json.load(open(a.out)) if os.path.exists(a.out) else {}
    for n in names:
        res[n] = run(n)
        print(n, res[n]["sizes"], res[n]["iterations"], res[n]["oracle_seconds"], "s", flush=True)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
