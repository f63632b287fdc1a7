"""Datalog front end (datalog.py): rules compiled to the engine's operator
program give the same relations as the hand-written drivers (programs.py,
which follow test/tc.cu, test/sg.cu and test/cspa.cu).  CPU: the oracle
engine."""
import os

import numpy as np
import pytest

import datalog as D
import programs as P
import workloads as W
from conftest import REF_ROOT
from gdlog_b200 import Engine

TC = """
path(x, y) :- edge(x, y).
path(x, z) :- path(x, y), edge(y, z).
"""

SG = """
sg(x, y) :- edge(p, x), edge(p, y), x != y.
sg(x, y) :- edge(a, x), sg(a, b), edge(b, y).
"""

# The rules of the CSPA driver (programs.cspa): the copies of its first LIE
# and the joins of its analysis LIE.
CSPA = """
vf(y, y) :- assign(x, y).
vf(x, x) :- assign(x, y).
vf(x, y) :- assign(x, y).
ma(y, y) :- assign(x, y).
ma(x, x) :- assign(x, y).
vf(x, y) :- vf(x, z), vf(z, y).
va(x, y) :- vf(z, x), vf(z, y).
vf(x, y) :- assign(x, z), ma(z, y).
ma(x, w) :- deref(y, x), va(y, z), deref(z, w).   % three atoms, a chain
va(x, y) :- vf(z, x), ma(z, w), vf(w, y).
"""


def sorted_rows(rel):
    r = rel.rows()
    return r[np.lexsort((r[:, 1], r[:, 0]))].tolist()


@pytest.mark.parametrize("edges", [lambda: W.grid_edges(10, 10), lambda: W.layered_dag(10, 8, 3),
                                   lambda: W.rmat_edges(7, 300, seed=5)])
def test_tc_rules_equal_the_driver(edges):
    e = edges()
    with Engine("oracle") as o:
        got = sorted_rows(D.run(o, TC, {"edge": e}).relations["path"])
    with Engine("oracle") as o:
        want = sorted_rows(P.tc(o, e).output)
    assert got == want


@pytest.mark.parametrize("seed", [1, 2])
def test_sg_rules_equal_the_driver(seed):
    e = W.rmat_edges(8, 600, seed=seed)
    with Engine("oracle") as o:
        got = sorted_rows(D.run(o, SG, {"edge": e}).relations["sg"])
    with Engine("oracle") as o:
        want = sorted_rows(P.sg(o, e).output)
    assert got == want


def test_cspa_rules_equal_the_driver():
    assign, deref = W.cspa_facts(120, 240, 90, seed=1)
    with Engine("oracle") as o:
        r = D.run(o, CSPA, {"assign": assign, "deref": deref})
        got = {k: sorted_rows(r.relations[k]) for k in ("vf", "ma", "va")}
    with Engine("oracle") as o:
        w = P.cspa(o, assign, deref)
        want = {"vf": sorted_rows(w.relations["value_flow"]),
                "ma": sorted_rows(w.relations["memory_alias"]),
                "va": sorted_rows(w.relations["value_alias"])}
    assert got == want


def test_components_in_dependency_order():
    rules = D.parse("a(x, y) :- e(x, y).  b(x, y) :- a(x, y).  b(x, z) :- b(x, y), a(y, z).")
    assert D._components(rules) == [["a"], ["b"]]


@pytest.mark.parametrize("bad", [
    "p(x, y) :- q(x, z).",                          # head variable not in the body
    "p(x, y) :- q(x, y), x != y.",                  # a Copy ignores predicates
    "p(x, y) :- q(x, a), r(b, y).",                 # no shared variable
    "p(x, y) :- q(x, a), r(a, b), s(b, c), t(c, y).",  # four atoms
    "p(x) :- q(x, y).",                             # not binary
])
def test_unsupported_rules_are_refused(bad):
    inputs = {k: np.zeros((0, 2), dtype=np.uint64) for k in "qrst"}
    with Engine("oracle") as o, pytest.raises(ValueError):
        D.run(o, bad, inputs)


@pytest.mark.gpu
def test_rules_on_the_gpu_engine():
    e = W.rmat_edges(8, 600, seed=2)
    g_edges = W.grid_edges(16, 16)
    with Engine("gpu") as g:
        sg_got = sorted_rows(D.run(g, SG, {"edge": e}, sync=g.sync).relations["sg"])
        g.clear()
        tc_got = sorted_rows(D.run(g, TC, {"edge": g_edges}, sync=g.sync).relations["path"])
    with Engine("oracle") as o:
        sg_want = sorted_rows(P.sg(o, e).output)
    with Engine("oracle") as o:
        tc_want = sorted_rows(P.tc(o, g_edges).output)
    assert sg_got == sg_want
    assert tc_got == tc_want


REF_SOUFFLE = os.path.join(REF_ROOT, "test", "souffle")


def write_facts(path, rows):
    with open(path, "w") as f:
        for a, b in np.asarray(rows).reshape(-1, 2).tolist():
            f.write(f"{a}\t{b}\n")


def test_program_file_with_directives(tmp_path):
    prog = tmp_path / "tc.dl"
    prog.write_text(""".decl edge(x: number, y: number)
.input edge
.decl path(x: number, y: number)
.output path
.printsize path
/* transitive closure */
path(x, y) :- edge(x, y).
path(x, z) :- path(x, y), edge(y, z).   // one step further
.decl hub(x: number, y: number)
.printsize hub
hub(x, x) :- edge(x, _).
""")
    e = W.layered_dag(6, 5, 2)
    write_facts(tmp_path / "edge.facts", e)
    with Engine("oracle") as o:
        res, sizes = D.run_file(o, str(prog), facts_dir=str(tmp_path), out_dir=str(tmp_path / "out"))
        got = sorted_rows(res.relations["path"])
    with Engine("oracle") as o:
        want = sorted_rows(P.tc(o, e).output)
    assert got == want and sizes["path"] == len(want)
    assert sizes["hub"] == len(np.unique(e[:, 0]))
    lines = open(tmp_path / "out" / "path.csv").read().split()
    assert len(lines) == 2 * len(want)


@pytest.mark.skipif(not os.path.isdir(REF_SOUFFLE), reason="reference programs not present")
def test_reference_souffle_programs_run(tmp_path):
    """The reference's own sg.dl and cspa.dl (test/souffle), their inputs
    from facts files, against the hand-written drivers."""
    e = W.rmat_edges(8, 600, seed=3)
    write_facts(tmp_path / "edge.facts", e)
    assign, deref = W.cspa_facts(120, 240, 90, seed=2)
    write_facts(tmp_path / "assign.facts", assign)
    write_facts(tmp_path / "dereference.facts", deref)
    with Engine("oracle") as o:
        res, sizes = D.run_file(o, os.path.join(REF_SOUFFLE, "sg.dl"), facts_dir=str(tmp_path))
        sg_got = sorted_rows(res.relations["sg"])
    with Engine("oracle") as o:
        assert sg_got == sorted_rows(P.sg(o, e).output)
    with Engine("oracle") as o:
        res, sizes = D.run_file(o, os.path.join(REF_SOUFFLE, "cspa.dl"), facts_dir=str(tmp_path))
        got = {k: sorted_rows(res.relations[k]) for k in ("ValueFlow", "MemoryAlias", "ValueAlias")}
    with Engine("oracle") as o:
        w = P.cspa(o, assign, deref)
        want = {"ValueFlow": sorted_rows(w.relations["value_flow"]),
                "MemoryAlias": sorted_rows(w.relations["memory_alias"]),
                "ValueAlias": sorted_rows(w.relations["value_alias"])}
    assert got == want
    assert sizes["ValueFlow"] == len(want["ValueFlow"])


@pytest.mark.skipif(not os.path.isdir(REF_SOUFFLE), reason="reference programs not present")
def test_reference_tc_program_runs(tmp_path):
    """The reference's tc.dl: closure by a rule whose two body atoms are
    both path (each one's DELTA against the other's FULL, a swapped mirror
    for the join on the first atom's second column); the same tuples as the
    linear driver, in fewer loop passes."""
    e = W.rmat_edges(7, 300, seed=5)
    write_facts(tmp_path / "edge.facts", e)
    with Engine("oracle") as o:
        res, sizes = D.run_file(o, os.path.join(REF_SOUFFLE, "tc.dl"), facts_dir=str(tmp_path))
        got = sorted_rows(res.relations["path"])
        passes = res.iterations["path"]
    with Engine("oracle") as o:
        w = P.tc(o, e)
        assert got == sorted_rows(w.output) and sizes["path"] == len(got)
        assert passes < w.iterations["tc"]


def test_command_line(tmp_path):
    import json
    import subprocess
    import sys
    prog = tmp_path / "sg.dl"
    prog.write_text(""".decl edge(x: number, y: number)
.input edge
.decl sg(x: number, y: number)
.output sg
.printsize sg
sg(x, y) :- edge(p, x), edge(p, y), x != y.
sg(x, y) :- edge(a, x), sg(a, b), edge(b, y).
""")
    e = W.rmat_edges(6, 120, seed=4)
    write_facts(tmp_path / "edge.facts", e)
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(here, "gdlog-multinode_b200", "datalog.py"),
                          str(prog), "--facts", str(tmp_path), "--out", str(tmp_path / "o"),
                          "--engine", "oracle"], capture_output=True, text=True, check=True)
    sizes = json.loads(out.stdout.strip().splitlines()[-1])["sizes"]
    with Engine("oracle") as o:
        want = P.sg(o, e).output.size()
    assert sizes["sg"] == want
    assert os.path.exists(tmp_path / "o" / "sg.csv")


PLEN = """
path(x, y, 1) :- edge(x, y).
path(x, y, l+1) :- edge(x, m), path(m, y, l).
"""


def test_path_length_rules_equal_the_driver():
    """Ternary path with a dependent length column (the shortest length of
    each pair), the length computed by l+1, the first lengths from a number
    in the head."""
    e = W.rmat_edges(7, 300, seed=6)
    with Engine("oracle", max_arity=3) as o:
        r = D.run(o, PLEN, {"edge": e}, deps={"path": 1})
        got = sorted(map(tuple, r.relations["path"].rows().tolist()))
    with Engine("oracle", max_arity=3) as o:
        want = sorted(map(tuple, P.path_length(o, e).output.rows().tolist()))
    assert got == want


@pytest.mark.skipif(not os.path.isdir(REF_SOUFFLE), reason="reference programs not present")
def test_reference_path_length_program_runs(tmp_path):
    e = W.layered_dag(8, 6, 4)
    write_facts(tmp_path / "edge.facts", e)
    with Engine("oracle", max_arity=3) as o:
        res, sizes = D.run_file(o, os.path.join(REF_SOUFFLE, "path_length.dl"),
                                facts_dir=str(tmp_path))
        got = sorted(map(tuple, res.relations["path"].rows().tolist()))
    with Engine("oracle", max_arity=3) as o:
        want = sorted(map(tuple, P.path_length(o, e).output.rows().tolist()))
    assert got == want and sizes["path"] == len(want)


def test_strata_and_mirrors():
    """A non-recursive component (sym) feeding a recursive one (reach) that
    joins on its second column (a swapped mirror kept by an ACopy), checked
    against a closure computed here."""
    prog = """
    sym(x, y) :- e(x, y).
    sym(x, y) :- e(y, x).
    reach(x, y) :- sym(x, y).
    reach(x, z) :- reach(x, y), sym(y, z).
    """
    e = W.rmat_edges(6, 60, seed=8)
    with Engine("oracle") as o:
        r = D.run(o, prog, {"e": e})
        got = set(map(tuple, r.relations["reach"].rows().tolist()))
        assert [k for k in r.iterations] == ["sym", "reach"]
    n = int(e.max()) + 1
    adj = np.zeros((n, n), dtype=bool)
    adj[e[:, 0].astype(int), e[:, 1].astype(int)] = True
    adj |= adj.T
    reach = adj.copy()
    while True:
        nxt = reach | ((reach.astype(np.int64) @ adj.astype(np.int64)) > 0)
        if (nxt == reach).all():
            break
        reach = nxt
    want = {(int(a), int(b)) for a, b in zip(*np.nonzero(reach))}
    assert got == want
