"""The engine's executable cache for loop graphs.

A program run again after Engine.clear() gets the same device blocks back
(the allocator replays the previous program's requests) and its loops take
the previous program's executable graphs, compared node by node, instead of
instantiating new ones.  Checked here: the second and later runs reuse the
executables; every run gives the golden (oracle) answer, including runs on
different data of the same shape, where the reused graph reads the new
relations; a different program does not take a graph it does not match;
GDLOG_NO_GRAPH_CACHE turns reuse off.
"""
import os
import subprocess
import sys

import pytest

import programs as P
import workloads as W
from gdlog_b200 import Engine
from test_oracle import GOLDEN, build_workload

pytestmark = pytest.mark.gpu


def summary(r):
    return ({k: v.size() for k, v in r.relations.items()},
            {k: hex(v.digest()) for k, v in r.relations.items()},
            r.iterations)


def reused(r):
    return [lie.stats()["graph_reused"] for lie in r.lies.values()]


@pytest.mark.parametrize("name", ["sg_rmat_s8_600_s1", "tc_grid_16x16", "cspa_v120_s1"])
@pytest.mark.parametrize("mode", ["dense", "sort", "dense_rows"])
def test_repeated_program_reuses_graphs(name, mode):
    prog, args = build_workload(name)
    want = GOLDEN["workloads"][name]
    flags = []
    with Engine("gpu", dedup=mode) as g:
        for _ in range(4):
            g.clear()
            r = prog(g, *args, sync=g.sync)
            sizes, digests, iters = summary(r)
            assert sizes == want["sizes"] and digests == want["digests"]
            assert iters == want["iterations"]
            flags.append(reused(r))
    assert not any(flags[0])
    # from the second repetition on every loop that launched a graph reuses it
    assert all(all(f) for f in flags[2:]), flags


def test_same_shape_new_data():
    """Different edges with the same row count and id domain: the graphs
    may be reused (they read the relations from device memory); every
    answer matches the oracle."""
    runs = [W.rmat_edges(9, 1500, seed=s) for s in (1, 2, 3, 1, 4)]
    got, flags = [], []
    with Engine("gpu") as g:
        for e in runs:
            g.clear()
            r = P.sg(g, e, sync=g.sync)
            got.append(summary(r))
            flags.append(reused(r))
    with Engine("oracle") as o:
        for e, have in zip(runs, got):
            assert summary(P.sg(o, e)) == have
    assert any(any(f) for f in flags[1:]), flags


def test_other_program_does_not_match():
    """TC after SG on the same engine: no graph of SG fits TC's loop."""
    e = W.rmat_edges(8, 600, seed=1)
    with Engine("gpu") as g:
        for _ in range(2):
            g.clear()
            P.sg(g, e, sync=g.sync)
        g.clear()
        r = P.tc(g, e, sync=g.sync)
        assert reused(r) == [0] * len(r.lies)
        with Engine("oracle") as o:
            assert summary(P.tc(o, e)) == summary(r)


def test_cache_can_be_turned_off():
    code = (
        "import programs as P, workloads as W\n"
        "from gdlog_b200 import Engine\n"
        "e = W.rmat_edges(8, 600, seed=1)\n"
        "with Engine('gpu') as g:\n"
        "    for _ in range(3):\n"
        "        g.clear(); r = P.sg(g, e, sync=g.sync)\n"
        "    print(sum(l.stats()['graph_reused'] for l in r.lies.values()))\n")
    env = dict(os.environ, GDLOG_NO_GRAPH_CACHE="1")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env["PYTHONPATH"] = os.pathsep.join([os.path.join(root, "gdlog-multinode_b200"),
                                         env.get("PYTHONPATH", "")])
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip().splitlines()[-1] == "0"
