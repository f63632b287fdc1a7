"""Pull-form joins (csrc/pull.cuh): joins into bitmaps whose output is
(outer column 1, inner column 1) gathered by output row from the transposed
outer.  Every case runs the pull form, the push form (k_join_bm) and the
oracle and compares sizes, digests, loop-pass counts and the per-iteration
(dedup, delta, full) log of src/lie.cu:193-197.

The domain sizes cover each layout of a unit of work: 2^8 ids (a unit of
256 transposed words spans 32 rows of 8 words), 2^12 (2 rows), 2^13 (one
row of 256 words), 2^14 (half a row) and 2^16 (an eighth of a row of 2048
words, the largest row)."""
import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import DELTA, FULL, INNER, NEWT, OUTER, PRED_NE, Engine

pytestmark = pytest.mark.gpu


def summarize(r):
    return {
        "sizes": {k: v.size() for k, v in r.relations.items()},
        "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
        "iterations": r.iterations,
        "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
    }


def three_ways(prog, *args):
    """The pull form, the push form and the oracle; the row-gather form
    (gathered along a static inner's in-edges, from 2^12 ids) must give the
    same as the pull form."""
    out = []
    for mode in ("dense_pull", "dense_push", "dense_rows"):
        with Engine("gpu", dedup=mode) as g:
            out.append(summarize(prog(g, *args, sync=g.sync)))
    with Engine("oracle") as o:
        out.append(summarize(prog(o, *args)))
    assert out[2] == out[0]
    return out[0], out[1], out[3]


@pytest.mark.parametrize("scale,edges", [(8, 600), (12, 5000), (13, 12000), (16, 3000)])
def test_sg_pull_matches_push_and_oracle(scale, edges):
    e = W.rmat_edges(scale, edges, seed=scale)
    assert int(e.max()) >= 1 << (scale - 1)
    pull, push, want = three_ways(P.sg, e)
    assert pull == want
    assert push == want


@pytest.mark.parametrize("case", ["grid_24", "dag_L30_W40", "rmat_s11"])
def test_tc_transposed_output_matches_push_and_oracle(case):
    """TC's join (edge FULL, path DELTA, output (inner 1, outer 1)) in the
    pull form with a transposed output folded into NEWT."""
    e = {"grid_24": lambda: W.grid_edges(24, 24),
         "dag_L30_W40": lambda: W.layered_dag(30, 40, 2),
         "rmat_s11": lambda: W.rmat_edges(11, 3000, seed=5)}[case]()
    pull, push, want = three_ways(P.tc, e)
    assert pull == want
    assert push == want


def test_sg_scale14_pull_equals_push():
    """The default bench workload (R-MAT scale 14, 40,000 edges)."""
    e = W.rmat_edges(14, 40000, seed=14)
    out = []
    for mode in ("dense_pull", "dense_push", "dense_rows", "dense"):
        with Engine("gpu", dedup=mode) as g:
            out.append(summarize(P.sg(g, e, sync=g.sync)))
    assert out[0] == out[1] == out[2] == out[3]
    assert out[0]["sizes"]["sg"] == 38069132


@pytest.mark.parametrize("v,seed", [(120, 1), (200, 4), (300, 3)])
def test_cspa_pull_matches_push_and_oracle(v, seed):
    """CSPA has six pull-shaped joins: DELTA outers of four relations, two
    tmp NEWT outers, FULL inners of update and static relations."""
    pull, push, want = three_ways(P.cspa, *W.cspa_facts(v, 2 * v, (3 * v) // 4, seed=seed))
    assert pull == want
    assert push == want


def test_cspa_1000_pull_equals_push():
    """A larger CSPA (beyond the oracle's memory: value_alias grows with the
    square of the variables): the join forms agree."""
    args = W.cspa_facts(1000, 2000, 750, seed=4)
    out = []
    for mode in ("dense_pull", "dense_push", "dense_rows"):
        with Engine("gpu", dedup=mode) as g:
            out.append(summarize(P.cspa(g, *args, sync=g.sync)))
    assert out[0] == out[1] == out[2]


@pytest.mark.parametrize("scale,edges", [(12, 9000), (13, 20000), (15, 60000)])
def test_sg_row_gather_matches_oracle(scale, edges):
    """Both of SG's recursive joins in the row-gather form (a DELTA outer and
    a tmp NEWT outer over the static edge relation), 2^12..2^15 ids."""
    e = W.rmat_edges(scale, edges, seed=scale + 1)
    with Engine("gpu", dedup="dense_rows") as g:
        got = summarize(P.sg(g, e, sync=g.sync))
    with Engine("gpu", dedup="dense_pull") as g:
        pull = summarize(P.sg(g, e, sync=g.sync))
    assert got == pull
    if scale <= 13:
        with Engine("oracle_bitset") as o:
            assert got == summarize(P.sg(o, e))


def rows_quirks(eng, sync=None):
    """Row-gather joins at the reference's edges, over 2^13 ids: a DELTA
    outer and a tmp NEWT outer over a static inner; the tmp NEWT also read
    by a push join (its list); an empty static inner zeroing a DELTA outer
    (src/join.cu:38-45) and another clearing a tmp NEWT outer."""
    rng = np.random.default_rng(9)
    a = eng.relation("a", index_flag=False)
    c = eng.relation("c", index_flag=False)
    e = eng.relation("e")
    z = eng.relation("z")
    t = eng.relation("t", index_flag=False, tmp_flag=True)
    u = eng.relation("u", index_flag=False, tmp_flag=True)
    eng.load(a, rng.integers(0, 6000, size=(2000, 2)).astype(np.uint64))
    eng.load(c, rng.integers(0, 6000, size=(500, 2)).astype(np.uint64))
    eng.load(e, rng.integers(0, 6000, size=(1500, 2)).astype(np.uint64))
    eng.load(z, None)
    eng.load(t, None)
    eng.load(u, None)
    lie = eng.lie()
    lie.add_relations(e, True)
    lie.add_relations(z, True)
    lie.add_relations(a, False)
    lie.add_relations(c, False)
    lie.add_tmp_relation(t)
    lie.add_tmp_relation(u)
    lie.add_join(e, FULL, a, DELTA, t, (OUTER(1), INNER(1)))    # t(b, x) :- a(k, b), e(k, x)
    lie.add_join(e, FULL, t, NEWT, a, (OUTER(1), INNER(1)))    # a(x, y) :- t(b, x), e(b, y)
    lie.add_join(e, FULL, t, NEWT, c, (OUTER(0), INNER(1)))    # push form: t's list
    lie.add_join(e, FULL, c, DELTA, u, (INNER(1), OUTER(1)))   # transposed output
    lie.add_join(z, FULL, u, NEWT, a, (OUTER(1), INNER(1)))    # empty inner: u cleared
    lie.add_join(z, FULL, c, DELTA, c, (OUTER(1), INNER(1)))   # empty inner: c's DELTA zeroed
    lie.max_iteration = 5
    it = lie.fixpoint()
    return it, a.size(), a.digest(), c.size(), c.digest(), lie.trace().tolist()


def static_outer_quirks(eng, sync=None):
    """Joins of two static FULLs in the row-gather form, over 2^13 ids: the
    predicate t[0] != t[1] in both column orders (inputs with self-loops, so
    diagonal candidates exist), output rows written directly and through a
    transposed twin, run once per fixpoint while a recursive join keeps the
    loop going, and an empty static inner that zeroes a static outer's
    count for the rest of the LIE (src/join.cu:38-45)."""
    rng = np.random.default_rng(13)
    e = eng.relation("e")
    f = eng.relation("f")
    z = eng.relation("z")
    s = eng.relation("s", index_flag=False)
    w = eng.relation("w", index_flag=False)
    ev = rng.integers(0, 5000, size=(3000, 2)).astype(np.uint64)
    ev[:200, 1] = ev[:200, 0]
    fv = rng.integers(0, 5000, size=(2500, 2)).astype(np.uint64)
    fv[:200, 1] = fv[:200, 0]
    eng.load(e, ev)
    eng.load(f, fv)
    eng.load(z, None)
    eng.load(s, None)
    eng.load(w, None)
    lie = eng.lie()
    lie.add_relations(e, True)
    lie.add_relations(f, True)
    lie.add_relations(z, True)
    lie.add_relations(s, False)
    lie.add_relations(w, False)
    lie.add_join(e, FULL, f, FULL, s, (INNER(1), OUTER(1)), pred=(PRED_NE, 0, 1))
    lie.add_join(f, FULL, e, FULL, w, (OUTER(1), INNER(1)), pred=(PRED_NE, 1, 0))
    lie.add_join(e, FULL, s, DELTA, s, (OUTER(1), INNER(1)))   # s(b, y) :- s(k, b), e(k, y)
    lie.add_join(z, FULL, f, FULL, w, (OUTER(1), INNER(1)))    # empty inner: f's count zeroed
    it = lie.fixpoint()
    return it, s.size(), s.digest(), w.size(), w.digest(), lie.trace().tolist()


def test_static_outer_row_gather_matches_oracle():
    got = []
    for mode in ("dense_rows", "dense_pull", "dense_push"):
        with Engine("gpu", dedup=mode) as g:
            got.append(static_outer_quirks(g))
    with Engine("oracle") as o:
        want = static_outer_quirks(o)
    assert got[0] == got[1] == got[2] == want


def test_row_gather_quirks_match_oracle():
    got = []
    for mode in ("dense_rows", "dense_pull", "dense_push"):
        with Engine("gpu", dedup=mode) as g:
            got.append(rows_quirks(g))
    with Engine("oracle") as o:
        want = rows_quirks(o)
    assert got[0] == want
    assert got[1] == want
    assert got[2] == want


def pull_quirks(eng, sync=None):
    """Pull-shaped joins at the reference's edges: an empty inner zeroes the
    outer's count (src/join.cu:38-45), for a DELTA and for a tmp NEWT outer;
    one tmp NEWT read by pull joins of both orientations and by a push join;
    ids >= 256 so the dense form runs over 2^9 ids."""
    rng = np.random.default_rng(5)
    base = rng.integers(0, 400, size=(300, 2)).astype(np.uint64)
    a = eng.relation("a")
    b = eng.relation("b")
    c = eng.relation("c")
    e = eng.relation("e")
    t = eng.relation("t", index_flag=False)
    eng.load(a, base[:150])
    eng.load(b, None)
    eng.load(c, np.array([[5, 6], [300, 7]], dtype=np.uint64))
    eng.load(e, base[150:])
    eng.load(t, None)
    lie = eng.lie()
    lie.add_relations(b, True)
    lie.add_relations(e, True)
    lie.add_relations(a, False)
    lie.add_relations(c, False)
    lie.add_tmp_relation(t)
    # t(y, z) :- a(x, y), e(x, z)         (pull: DELTA outer)
    lie.add_join(e, FULL, a, DELTA, t, (OUTER(1), INNER(1)))
    # a(y, z) :- t(x, y), e(x, z)         (pull: tmp NEWT outer)
    lie.add_join(e, FULL, t, NEWT, a, (OUTER(1), INNER(1)))
    # c(z, y) :- t(x, y), e(x, z)         (pull, transposed output: same tmp NEWT)
    lie.add_join(e, FULL, t, NEWT, c, (INNER(1), OUTER(1)))
    # c(z, y) :- t(x, y), e(x, z), z != y  (push: a predicate)
    lie.add_join(e, FULL, t, NEWT, c, (INNER(1), OUTER(1)), pred=(PRED_NE, 0, 1))
    # a(z, y) :- a(x, y), a(x, z)         (pull, transposed output; FULL inner
    #                                      of an update relation: row-OR)
    lie.add_join(a, FULL, a, DELTA, a, (INNER(1), OUTER(1)))
    # c(y, z) :- t(x, y), b(x, z)         (pull, empty inner: t's count zeroed)
    lie.add_join(b, FULL, t, NEWT, c, (OUTER(1), INNER(1)))
    # c(y, z) :- t(x, y), e(x, z)         (pull: sees t emptied)
    lie.add_join(e, FULL, t, NEWT, c, (OUTER(1), INNER(1)))
    # c(y, z) :- c(x, y), b(x, z)         (pull, empty inner: c's DELTA zeroed)
    lie.add_join(b, FULL, c, DELTA, c, (OUTER(1), INNER(1)))
    lie.max_iteration = 6
    it = lie.fixpoint()
    return it, a.size(), a.digest(), c.size(), c.digest(), lie.trace().tolist()


def test_pull_quirks_match_oracle():
    got = []
    for mode in ("dense_pull", "dense_push"):
        with Engine("gpu", dedup=mode) as g:
            got.append(pull_quirks(g))
    with Engine("oracle") as o:
        want = pull_quirks(o)
    assert got[0] == want
    assert got[1] == want


def test_pull_graph_and_stream_paths_agree(monkeypatch):
    e = W.rmat_edges(10, 4096, seed=14)
    out = []
    for no_graph in (False, True):
        if no_graph:
            monkeypatch.setenv("GDLOG_NO_GRAPH", "1")
        with Engine("gpu", dedup="dense_pull") as g:
            out.append(summarize(P.sg(g, e, sync=g.sync)))
    assert out[0] == out[1]


def test_pull_form_is_what_runs():
    """With the pull form on, each of SG's two recursive joins is one launch
    per iteration (k_join_pull_bm) instead of two (k_join_bm and its heavy
    pieces), so the join family launches less with the same results."""
    e = W.rmat_edges(10, 4096, seed=14)
    joins = {}
    for mode in ("dense_pull", "dense_push"):
        with Engine("gpu", dedup=mode) as g:
            g.set_profile(True)
            g.profile_reset()
            r = P.sg(g, e, sync=g.sync)
            g.set_profile(False)
            joins[mode] = (g.profile()["join_mat"]["launches"], r.iterations["sg"])
    (pull_l, it), (push_l, it2) = joins["dense_pull"], joins["dense_push"]
    assert it == it2
    # the init LIE's join (push in both) plus 2 or 4 launches per pass
    assert push_l - pull_l == 2 * it


def test_delta_left_by_max_iteration_is_listed():
    """A DELTA read only through its transposed bitmap is not listed during
    the loop; when max_iteration ends the loop with a DELTA left, its list
    is written afterwards (set_reload_full(False) keeps it)."""
    e = W.rmat_edges(10, 4096, seed=3)

    def prog(eng):
        edge = eng.relation("edge")
        sg = eng.relation("sg", index_flag=False)
        tmp = eng.relation("tmp", index_flag=False)
        eng.load(edge, e)
        eng.load(sg, e)
        eng.load(tmp, None)
        lie = eng.lie()
        lie.set_reload_full(False)
        lie.add_relations(edge, True)
        lie.add_relations(sg, False)
        lie.add_tmp_relation(tmp)
        lie.add_join(edge, FULL, sg, DELTA, tmp, (OUTER(1), INNER(1)))
        lie.add_join(edge, FULL, tmp, NEWT, sg, (OUTER(1), INNER(1)))
        lie.max_iteration = 2
        it = lie.fixpoint()
        return (it, sg.size(), sg.digest(), sg.size(DELTA), sg.digest(DELTA),
                lie.trace().tolist())

    got = []
    for mode in ("dense_pull", "dense_push"):
        with Engine("gpu", dedup=mode) as g:
            got.append(prog(g))
    with Engine("oracle") as o:
        want = prog(o)
    assert want[3] > 0
    assert got[0] == want
    assert got[1] == want
