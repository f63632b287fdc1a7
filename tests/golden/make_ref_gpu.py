"""Run the reference CUDA engine (oracle/_ref/ref_runner, built from the
reference's own sources by `make -C oracle ref`) on the synthetic workloads
and record its answers as fixtures (tests/golden/ref_gpu.json).

Needs a CUDA device.  Usage, from the repository root:

    python tests/golden/make_ref_gpu.py --out tests/golden/ref_gpu.json \
        [--only NAME[,NAME...]] [--timeout SECONDS]

The points-to analysis stops at 300 variables here: the reference engine
made an illegal memory access (its src/join.cu:120) on the 2,000-variable
input and ran out of device memory on the 6,000-variable one, so it is not
run on those again; the bit-matrix oracle pins them instead
(tests/golden/make_cspa_large.py).

For each workload it writes the TSV inputs the reference drivers read
(test/tc.cu:31-57 format), runs the runner, and stores the sizes, loop-pass
counts, digests of the sorted FULL tuples and the wall seconds of the
fixpoint loops.  The tests compare these with the engine's answers.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "gdlog-multinode_b200"))

import workloads as W  # noqa: E402

RUNNER = os.path.join(REPO, "oracle", "_ref", "ref_runner")

WORKLOADS = {
    "tc_grid_16x16": ("tc", lambda: (W.grid_edges(16, 16),)),
    "tc_grid_64x64": ("tc", lambda: (W.grid_edges(64, 64),)),
    "tc_dag_L12_W10_s1": ("tc", lambda: (W.layered_dag(12, 10, 1),)),
    "sg_rmat_s8_600_s1": ("sg", lambda: (W.rmat_edges(8, 600, seed=1),)),
    "sg_rmat_s10_4096_s14": ("sg", lambda: (W.rmat_edges(10, 4096, seed=14),)),
    "sg_rmat_s14_40000_s14": ("sg", lambda: (W.rmat_edges(14, 40000, seed=14),)),
    "cspa_v120_s1": ("cspa", lambda: W.cspa_facts(120, 240, 90, seed=1)),
    "cspa_v300_s3": ("cspa", lambda: W.cspa_facts(300, 600, 225, seed=3)),
    "plen_grid_16x16": ("plen", lambda: (W.grid_edges(16, 16),)),
    "plen_grid_64x64": ("plen", lambda: (W.grid_edges(64, 64),)),
    "plen_dag_L12_W10_s1": ("plen", lambda: (W.layered_dag(12, 10, 1),)),
    "plen_rmat_s8_600_s1": ("plen", lambda: (W.rmat_edges(8, 600, seed=1),)),
}


def run(name: str, timeout: float) -> dict:
    prog, make = WORKLOADS[name]
    inputs = make()
    with tempfile.TemporaryDirectory() as d:
        files = []
        for i, rows in enumerate(inputs):
            p = os.path.join(d, f"in{i}.tsv")
            W.write_tsv(p, rows)
            files.append(p)
        try:
            r = subprocess.run([RUNNER, prog, *files], stdout=subprocess.DEVNULL,
                               stderr=subprocess.PIPE, text=True, timeout=timeout)
        except subprocess.TimeoutExpired:
            return {"error": f"timed out after {timeout} s"}
    line = [ln for ln in r.stderr.splitlines() if ln.startswith("REF ")]
    if r.returncode != 0 or not line:
        return {"error": f"exit {r.returncode}: {r.stderr[-400:]}"}
    return json.loads(line[-1][4:])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_gpu.json"))
    ap.add_argument("--only", default="")
    ap.add_argument("--timeout", type=float, default=600)
    a = ap.parse_args()
    names = a.only.split(",") if a.only else list(WORKLOADS)
    res = {}
    if os.path.exists(a.out):
        res = json.load(open(a.out))
    for n in names:
        res[n] = run(n, a.timeout)
        print(n, res[n], flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
