"""CPU tests of the oracle (test infrastructure) and of the host-side logic.

Pins the oracle before it is trusted as the checker:
  * the analytic closure of the 64x64 grid (4,322,304 tuples, 126 loop
    passes of the left-linear program test/tc.cu:131-133);
  * the same-generation sizes the reference publishes (README.md:80-103,
    test/cuDF/sg.json) on the reference's own data files, when those files
    are present on this machine;
  * the committed golden fixtures (tests/golden/golden.json, written by
    tests/golden/make_golden.py) for every small workload.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import DELTA, FULL, INNER, NEWT, OUTER, PRED_NE, SRC, Engine, digest_rows

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))
from conftest import REF_ROOT

REF_DATA = os.path.join(REF_ROOT, "data")

SMALL = [k for k, v in GOLDEN["workloads"].items() if v["oracle_seconds"] < 2.0]


def build_workload(name):
    """Rebuild the inputs of a golden workload from its name."""
    parts = name.split("_")
    if name.startswith("tc_grid_"):
        r, c = map(int, parts[2].split("x"))
        return P.tc, (W.grid_edges(r, c),)
    if name.startswith("tc_dag_"):
        L, Wd, s = int(parts[2][1:]), int(parts[3][1:]), int(parts[4][1:])
        return P.tc, (W.layered_dag(L, Wd, s),)
    if name.startswith("sg_rmat_"):
        scale, n, s = int(parts[2][1:]), int(parts[3]), int(parts[4][1:])
        return P.sg, (W.rmat_edges(scale, n, seed=s),)
    if name.startswith("cspa_v"):
        v, s = int(parts[1][1:]), int(parts[2][1:])
        return P.cspa, W.cspa_facts(v, 2 * v, (3 * v) // 4, seed=s)
    raise KeyError(name)


def run_program(kind, name):
    prog, args = build_workload(name)
    eng = Engine(kind)
    r = prog(eng, *args)
    out = {
        "sizes": {k: v.size() for k, v in r.relations.items()},
        "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
        "iterations": r.iterations,
        "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
    }
    eng.close()
    return out


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_golden(oracle_lib, name):
    got = run_program("oracle", name)
    want = GOLDEN["workloads"][name]
    assert got["sizes"] == want["sizes"]
    assert got["iterations"] == want["iterations"]
    assert got["digests"] == want["digests"]
    assert got["traces"] == want["traces"]


def test_grid_tc_analytic(oracle_lib):
    """64x64 grid: (64*65/2)^2 - 4096 pairs, found at iteration d-2 for
    Manhattan distance d, so 126 loop passes including the empty one."""
    assert W.grid_tc_size(64, 64) == 4322304
    g = GOLDEN["workloads"]["tc_grid_64x64"]
    assert g["sizes"]["path"] == 4322304
    assert g["iterations"]["tc"] == 126
    with Engine("oracle") as eng:
        r = P.tc(eng, W.grid_edges(64, 64))
        assert r.output.size() == 4322304
        assert r.iterations["tc"] == 126
        assert hex(r.output.digest()) == g["digests"]["path"]


def test_grid_small_closure_bruteforce(oracle_lib):
    """Closure of a 6x5 grid equals reachability computed by plain BFS."""
    e = W.grid_edges(6, 5)
    n = 30
    adj = [[] for _ in range(n)]
    for u, v in e.tolist():
        adj[u].append(v)
    want = set()
    for s in range(n):
        seen, stack = set(), [s]
        while stack:
            u = stack.pop()
            for v in adj[u]:
                if v not in seen:
                    seen.add(v)
                    stack.append(v)
        want |= {(s, v) for v in seen}
    with Engine("oracle") as eng:
        r = P.tc(eng, e)
        got = {tuple(x) for x in r.output.rows().tolist()}
    assert got == want
    assert len(want) == W.grid_tc_size(6, 5)


def sg_bruteforce(edges):
    """sg(x,y) :- edge(p,x), edge(p,y), x!=y.  sg(x,y) :- edge(a,x), sg(a,b),
    edge(b,y).  Naive evaluation to a fixpoint (test/souffle/sg.dl)."""
    out = {}
    for u, v in edges.tolist():
        out.setdefault(u, set()).add(v)
    sg = {(x, y) for p in out for x in out[p] for y in out[p] if x != y}
    while True:
        new = {(x, y) for (a, b) in sg for x in out.get(a, ()) for y in out.get(b, ())}
        if new <= sg:
            return sg
        sg |= new


@pytest.mark.parametrize("seed", [1, 2])
def test_sg_bruteforce(oracle_lib, seed):
    e = W.rmat_edges(6, 120, seed=seed)
    with Engine("oracle") as eng:
        r = P.sg(eng, e)
        got = {tuple(x) for x in r.output.rows().tolist()}
    assert got == sg_bruteforce(e)


def cspa_bruteforce(assign, deref):
    """test/souffle/cspa.dl:25-39, naive evaluation."""
    a = {tuple(x) for x in assign.tolist()}
    d = {tuple(x) for x in deref.tolist()}
    vf = {(y, x) for (y, x) in a} | {(x, x) for (x, _) in a} | {(x, x) for (_, x) in a}
    ma = {(x, x) for (x, _) in a} | {(x, x) for (_, x) in a}
    va = set()
    while True:
        n_vf = set(vf)
        n_vf |= {(x, y) for (x, z) in a for (z2, y) in ma if z == z2}
        n_vf |= {(x, y) for (x, z) in vf for (z2, y) in vf if z == z2}
        n_ma = set(ma)
        n_ma |= {(x, w) for (y, x) in d for (y2, z) in va if y == y2 for (z2, w) in d if z == z2}
        n_va = set(va)
        n_va |= {(x, y) for (z, x) in vf for (z2, y) in vf if z == z2}
        n_va |= {(x, y) for (z, x) in vf for (z2, w) in ma if z == z2
                 for (w2, y) in vf if w == w2}
        if n_vf == vf and n_ma == ma and n_va == va:
            return vf, ma, va
        vf, ma, va = n_vf, n_ma, n_va


def test_cspa_bruteforce(oracle_lib):
    assign, deref = W.cspa_facts(30, 50, 20, seed=5)
    vf, ma, va = cspa_bruteforce(assign, deref)
    with Engine("oracle") as eng:
        r = P.cspa(eng, assign, deref)
        got = {k: {tuple(x) for x in v.rows().tolist()} for k, v in r.relations.items()}
    assert got["value_flow"] == vf
    assert got["memory_alias"] == ma
    assert got["value_alias"] == va


@pytest.mark.parametrize("fname", sorted(GOLDEN["published_sg"]))
def test_published_sg_sizes(oracle_lib, fname):
    """The oracle reproduces the SG sizes the reference publishes."""
    rec = GOLDEN["published_sg"][fname]
    assert rec["oracle"]["size"] == rec["published_size"]
    path = os.path.join(REF_DATA, fname)
    if not os.path.exists(path) or os.path.getsize(path) > 2_000_000:
        pytest.skip("reference data file not on this machine")
    data = open(path, "rb").read()
    assert hashlib.sha256(data).hexdigest() == rec["sha256"]
    with Engine("oracle") as eng:
        r = P.sg(eng, W.read_tsv(path))
        assert r.output.size() == rec["published_size"]
        assert r.iterations == rec["oracle"]["iterations"]


def test_digest_restatement(oracle_lib):
    rows = np.array([[0, 1], [0, 5], [3, 2]], dtype=np.uint64)
    with Engine("oracle") as eng:
        rel = eng.relation("x")
        eng.load(rel, rows[::-1].copy())
        assert rel.digest() == digest_rows(rows)
        assert rel.rows().tolist() == rows.tolist()


def test_workload_shapes():
    assert len(W.grid_edges(64, 64)) == 8064
    e = W.rmat_edges(14, 40000, seed=14)
    assert len(e) == 40000
    assert (e[:, 0] != e[:, 1]).all()
    assert len(np.unique(e[:, 0] * 2**32 + e[:, 1])) == 40000
    assert e.max() < 2**14
    a, d = W.cspa_facts()
    assert a.shape == (40000, 2) and d.shape == (15000, 2)
    assert a.max() < 20000 and d.max() < 20000
    dag = W.layered_dag(5, 7, 1)
    assert ((dag[:, 1] // 7) == (dag[:, 0] // 7) + 1).all()
    batch = W.dag_batch(16)
    assert all(8 <= L <= 128 and 16 <= Wd <= 256 for L, Wd, _ in batch)


def test_reference_cuda_build_agrees_with_oracle():
    """The reference's own CUDA engine (compiled unmodified from its
    sources, run on a B200 by tests/golden/make_ref_gpu.py) gives the same
    sizes, loop-pass counts and digests of the sorted result as the
    oracle's golden fixtures."""
    path = os.path.join(HERE, "golden", "ref_gpu.json")
    ref = json.load(open(path))
    checked = 0
    for name, rec in ref.items():
        if "error" in rec or name not in GOLDEN["workloads"]:
            continue
        want = GOLDEN["workloads"][name]
        assert rec["sizes"] == want["sizes"], name
        assert rec["iterations"] == want["iterations"], name
        assert rec["digests"] == want["digests"], name
        assert rec["sorted"], name
        checked += 1
    assert checked >= 4
