"""Arity 3 with a dependent column: the reference's path_length program
(test/path_length.cu:59-140; path(a, y, l + 1) :- edge(a, x), path(x, y, l),
a pair (a, y) new only while no path(a, y, _) exists).

The oracle is pinned by a restatement of what that program computes -- every
pair reachable by at least one edge, with its shortest length in edges
(breadth-first search below) -- and by the reference engine's own answers
(tests/golden/ref_gpu.json, oracle/ref_runner.cu's "plen" program run on a
B200).  The CUDA engine is compared with both, bit-exact."""
import collections
import json
import os

import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import (DELTA, FULL, INNER, OUTER, PLUS, Engine, GdlError, digest_rows)

HERE = os.path.dirname(os.path.abspath(__file__))
REF_GPU = json.load(open(os.path.join(HERE, "golden", "ref_gpu.json")))

CASES = {
    "plen_grid_16x16": lambda: W.grid_edges(16, 16),
    "plen_dag_L12_W10_s1": lambda: W.layered_dag(12, 10, 1),
    "plen_rmat_s8_600_s1": lambda: W.rmat_edges(8, 600, seed=1),
}


def shortest_paths(edges):
    """{(a, y): d} for every y reachable from a by >= 1 edge, d the fewest edges."""
    adj = collections.defaultdict(list)
    for a, b in np.asarray(edges).tolist():
        adj[a].append(b)
    out = {}
    for a in list(adj):
        dist = {}
        q = collections.deque((b, 1) for b in adj[a])
        while q:
            v, d = q.popleft()
            if v in dist:
                continue
            dist[v] = d
            for w in adj[v]:
                if w not in dist:
                    q.append((w, d + 1))
        for y, d in dist.items():
            out[(a, y)] = d
    return out


def run(kind, edges):
    with Engine(kind, max_arity=3) as eng:
        r = P.path_length(eng, edges, sync=getattr(eng, "sync", None))
        rows = r.relations["path"].rows()
        return rows, r.relations["path"].digest(), dict(r.iterations)


@pytest.mark.parametrize("name", ["plen_grid_16x16", "plen_dag_L12_W10_s1", "plen_rmat_s8_600_s1"])
def test_oracle_gives_shortest_lengths(name):
    edges = np.unique(CASES[name](), axis=0)
    rows, dig, _ = run("oracle", edges)
    want = shortest_paths(edges)
    got = {(a, y): l for a, y, l in rows.tolist()}
    assert len(got) == len(rows) and got == want
    assert dig == digest_rows(rows)


@pytest.mark.parametrize("name", ["plen_grid_16x16", "plen_dag_L12_W10_s1", "plen_rmat_s8_600_s1"])
def test_oracle_matches_reference_engine(name):
    ref = REF_GPU.get(name)
    if not ref or "sizes" not in ref:
        pytest.skip("reference answer not recorded")
    rows, dig, it = run("oracle", CASES[name]())
    assert ref["sizes"]["path"] == len(rows)
    assert ref["digests"]["path"] == hex(dig)
    assert ref["iterations"]["plen"] == it["plen"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["plen_grid_16x16", "plen_dag_L12_W10_s1", "plen_rmat_s8_600_s1"])
def test_gpu_matches_oracle(name):
    edges = CASES[name]()
    g = run("gpu", edges)
    o = run("oracle", edges)
    assert (g[0] == o[0]).all() and g[1] == o[1] and g[2] == o[2]


@pytest.mark.gpu
def test_gpu_64x64_grid_lengths():
    """Full-size grid: 4,322,304 pairs, each with its Manhattan length."""
    rows, dig, it = run("gpu", W.grid_edges(64, 64))
    assert len(rows) == 4322304
    a, y, l = rows[:, 0].astype(np.int64), rows[:, 1].astype(np.int64), rows[:, 2].astype(np.int64)
    assert (l == np.abs(y // 64 - a // 64) + np.abs(y % 64 - a % 64)).all()
    _, dig_o, it_o = run("oracle", W.grid_edges(64, 64))
    assert dig == dig_o and it == it_o
    ref = REF_GPU["plen_grid_64x64"]  # the reference engine's own answer
    assert hex(dig) == ref["digests"]["path"] and it["plen"] == ref["iterations"]["plen"]


@pytest.mark.gpu
def test_arity3_load_export_and_limits(tmp_path):
    rows = np.array([[5, 7, 2], [1, 2, 3], [5, 7, 1], [1, 2, 3]], dtype=np.uint64)
    with Engine("gpu") as g:
        r = g.relation("r3", arity=3, dependent_column_size=1)
        g.load(r, rows)
        assert r.rows().tolist() == [[1, 2, 3], [5, 7, 1], [5, 7, 2]]
        n = r.dump_tsv(str(tmp_path / "r3.tsv"))
        assert n == 3 and (tmp_path / "r3.tsv").read_text() == "1\t2\t3\n5\t7\t1\n5\t7\t2\n"
        # ids below 2^3 fixed column 2 at 32 - 3 = 29 bits: a larger id is refused
        with pytest.raises(GdlError):
            g.load(r, np.array([[1 << 30, 0, 0]], dtype=np.uint64))


@pytest.mark.gpu
def test_generated_value_too_large_fails_cleanly():
    """Ids near 2^30 leave column 2 one bit; a length-2 path does not fit and
    the fixpoint fails with a status instead of storing a wrong tuple."""
    big = (1 << 30) + 5
    edges = np.array([[0, 1], [1, big]], dtype=np.uint64)
    with Engine("gpu") as g:
        with pytest.raises(GdlError) as ei:
            P.path_length(g, edges, sync=g.sync)
        assert "too large" in str(ei.value) or "below 2^" in str(ei.value)
