"""CPU tests of the bit-matrix oracle (oracle/oracle_bitset.cpp, test
infrastructure), which produces the large points-to fixture
(tests/golden/cspa_large.json) that the CUDA engine is checked against.

It is pinned before it is trusted:
  * against the list oracle's committed answers (tests/golden/golden.json,
    whole per-iteration traces included) on every small workload;
  * against the reference CUDA build's own answers (tests/golden/ref_gpu.json,
    recorded by tests/golden/make_ref_gpu.py) where they exist, including the
    64x64 grid closure and same generation on R-MAT scale 14;
  * against the list oracle run here on the reference's semantic quirks:
    an empty inner, an empty Copy source, predicates, duplicated and
    unsorted input, max_iteration, reload_full off and repeated fixpoints;
  * and the committed mid-size points-to fixtures are re-derived here.
"""
import json
import os

import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import (DELTA, FULL, INNER, NEWT, OUTER, PRED_GE, PRED_GT, PRED_LT, PRED_NE, SRC,
                        Engine, GdlError)
from test_oracle import GOLDEN, build_workload

HERE = os.path.dirname(os.path.abspath(__file__))
REF_GPU = json.load(open(os.path.join(HERE, "golden", "ref_gpu.json")))
LARGE = json.load(open(os.path.join(HERE, "golden", "cspa_large.json")))


def summarize(r):
    return {
        "sizes": {k: v.size() for k, v in r.relations.items()},
        "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
        "iterations": dict(r.iterations),
        "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
    }


ARITY2 = [k for k in GOLDEN["workloads"] if not k.startswith("plen")]


@pytest.mark.parametrize("name", ARITY2)
def test_bitset_oracle_matches_list_oracle_golden(name):
    prog, args = build_workload(name)
    with Engine("oracle_bitset") as e:
        got = summarize(prog(e, *args))
    want = GOLDEN["workloads"][name]
    assert got["sizes"] == want["sizes"]
    assert got["iterations"] == want["iterations"]
    assert got["digests"] == want["digests"]
    assert got["traces"] == want["traces"]


REF_CASES = {
    "tc_grid_64x64": (P.tc, lambda: (W.grid_edges(64, 64),)),
    "sg_rmat_s10_4096_s14": (P.sg, lambda: (W.rmat_edges(10, 4096, seed=14),)),
    "sg_rmat_s14_40000_s14": (P.sg, lambda: (W.rmat_edges(14, 40000, seed=14),)),
    "cspa_v300_s3": (P.cspa, lambda: W.cspa_facts(300, 600, 225, seed=3)),
}


@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_bitset_oracle_matches_reference_cuda_build(name):
    if name not in REF_GPU or "sizes" not in REF_GPU[name]:
        pytest.skip(f"no answer of the reference CUDA build recorded for {name}")
    prog, make = REF_CASES[name]
    with Engine("oracle_bitset") as e:
        got = summarize(prog(e, *make()))
    want = REF_GPU[name]
    assert got["sizes"] == want["sizes"]
    assert got["digests"] == want["digests"]
    assert got["iterations"] == want["iterations"]


@pytest.mark.parametrize("name", ["cspa_v2000_s3", "cspa_v6000_s3"])
def test_large_cspa_fixture_rederived(name):
    from golden.make_cspa_large import WORKLOADS
    with Engine("oracle_bitset") as e:
        got = summarize(P.cspa(e, *WORKLOADS[name]()))
    want = LARGE[name]
    for k in ("sizes", "digests", "iterations", "traces"):
        assert got[k] == want[k], k


def test_large_cspa_fixture_self_consistent():
    """The C3 fixture's traces end where its sizes say, and every pass's
    FULL is the previous FULL plus its DELTA."""
    c3 = LARGE["cspa_c3"]
    assert c3["inputs"] == {"assign_rows": 40000, "dereference_rows": 15000}
    tr = np.array(c3["traces"]["analysis"], dtype=np.uint64)
    ids = sorted(set(tr[:, 1].tolist()))
    last = {}
    for it, rid, dedup, delta, full in tr.tolist():
        prev = last.get(rid)
        if prev is not None:
            assert full == prev + delta
        last[rid] = full
    assert tr[:, 0].max() + 1 == c3["iterations"]["analysis"]
    fulls = sorted(last[r] for r in ids)
    for v in c3["sizes"].values():
        assert v in fulls


# -- the reference's quirks, against the list oracle run here ---------------

def quirk_empty_inner(eng):
    a = eng.relation("a")
    b = eng.relation("b")
    c = eng.relation("c")
    eng.load(a, np.array([[1, 2], [2, 3], [3, 4]], dtype=np.uint64))
    eng.load(b, None)
    eng.load(c, np.array([[5, 6]], dtype=np.uint64))
    lie = eng.lie()
    lie.add_relations(b, True)
    lie.add_relations(a, False)
    lie.add_relations(c, False)
    lie.add_join(b, FULL, a, DELTA, a, (INNER(1), OUTER(1)))
    lie.add_copy(a, DELTA, c, (SRC(1), SRC(0)))
    lie.add_join(a, FULL, a, DELTA, c, (OUTER(0), INNER(1)))
    it = lie.fixpoint()
    return it, a.size(), c.size(), c.digest(), lie.trace().tolist()


def quirk_full_zeroed(eng):
    """An empty inner zeroes an outer FULL; the next flush restores it."""
    e = W.rmat_edges(6, 150, seed=4)
    edge = eng.relation("edge")
    none = eng.relation("none")
    path = eng.relation("path", index_flag=False)
    eng.load(edge, W.reverse(e))
    eng.load(none, None)
    eng.load(path, e)
    lie = eng.lie()
    lie.add_relations(edge, True)
    lie.add_relations(none, True)
    lie.add_relations(path, False)
    lie.add_join(none, FULL, path, FULL, path, (INNER(1), OUTER(1)))
    lie.add_join(edge, FULL, path, DELTA, path, (INNER(1), OUTER(1)))
    it = lie.fixpoint()
    return it, path.size(), path.digest(), lie.trace().tolist()


def quirk_generic_hooks(eng):
    """Column selections other than (inner 1, outer 1), and predicates the
    bit-matrix product does not special-case."""
    e = W.rmat_edges(7, 400, seed=11)
    edge = eng.relation("edge")
    out = [eng.relation(f"o{i}", index_flag=False) for i in range(5)]
    eng.load(edge, e)
    for r in out:
        eng.load(r, None)
    lie = eng.lie()
    lie.add_relations(edge, True)
    for r in out:
        lie.add_relations(r, False)
    lie.add_join(edge, FULL, edge, FULL, out[0], (OUTER(0), INNER(1)))
    lie.add_join(edge, FULL, edge, FULL, out[1], (INNER(1), INNER(1)))
    lie.add_join(edge, FULL, edge, FULL, out[2], (INNER(1), OUTER(1)), pred=(PRED_LT, 0, 1))
    lie.add_join(edge, FULL, edge, FULL, out[3], (OUTER(1), INNER(1)), pred=(PRED_GE, 1, 0))
    lie.add_copy(edge, FULL, out[4], (SRC(1), SRC(1)))
    lie.add_join(edge, FULL, out[4], DELTA, out[4], (INNER(0), OUTER(0)))
    it = lie.fixpoint()
    return it, [(r.size(), r.digest()) for r in out], lie.trace().tolist()


def quirk_duplicates_and_raw_delta(eng):
    """DELTA at loop start is the first |FULL| raw rows in load order, so a
    duplicated input row leaves a distinct row out of it."""
    e = np.array([[3, 4], [1, 2], [3, 4], [2, 3], [4, 5], [0, 1]], dtype=np.uint64)
    edge = eng.relation("edge")
    path = eng.relation("path", index_flag=False)
    eng.load(edge, W.reverse(e))
    eng.load(path, e)
    lie = eng.lie()
    lie.set_reload_full(False)
    lie.add_relations(edge, True)
    lie.add_relations(path, False)
    lie.add_join(edge, FULL, path, DELTA, path, P.REORDER_PATH)
    it = lie.fixpoint()
    return it, path.size(), path.digest(), lie.trace().tolist()


def quirk_cap_and_repeat(eng):
    """max_iteration, reload_full off, then a second LIE over the result."""
    e = W.grid_edges(9, 9)
    res = []
    edge = eng.relation("edge")
    path = eng.relation("path", index_flag=False)
    eng.load(edge, W.reverse(e))
    eng.load(path, e)
    for cap, reload in ((3, False), (1000, True), (1000, True)):
        lie = eng.lie()
        lie.set_reload_full(reload)
        lie.add_relations(edge, True)
        lie.add_relations(path, False)
        lie.add_join(edge, FULL, path, DELTA, path, P.REORDER_PATH)
        lie.max_iteration = cap
        it = lie.fixpoint()
        res.append((it, path.size(), path.digest(), lie.trace().tolist()))
    return res


def quirk_acopy_and_tmp(eng):
    """SG's recursive shape with the tmp relation read as NEWT, and an ACopy
    mirror of a NEWT that empties."""
    e = W.rmat_edges(7, 500, seed=5)
    r = P.sg(eng, e)
    edge = eng.relation("e2")
    m = eng.relation("mirror")
    eng.load(edge, e)
    eng.load(m, None)
    lie = eng.lie()
    lie.add_relations(edge, False)
    lie.add_relations(m, False)
    lie.add_join(edge, FULL, edge, DELTA, edge, (INNER(1), OUTER(1)), pred=(PRED_NE, 0, 1))
    lie.add_acopy(edge, m, (SRC(1), SRC(0)))
    it = lie.fixpoint()
    return (summarize(r), it, edge.size(), edge.digest(), m.size(), m.digest(),
            lie.trace().tolist())


@pytest.mark.parametrize("prog", [quirk_empty_inner, quirk_full_zeroed, quirk_generic_hooks,
                                  quirk_duplicates_and_raw_delta, quirk_cap_and_repeat,
                                  quirk_acopy_and_tmp])
def test_bitset_oracle_quirks_match_list_oracle(prog):
    with Engine("oracle") as o:
        want = prog(o)
    with Engine("oracle_bitset") as b:
        got = prog(b)
    assert got == want


@pytest.mark.parametrize("kind", [PRED_NE, PRED_GT])
def test_bitset_oracle_predicates(kind):
    e = W.rmat_edges(8, 700, seed=12)

    def prog(eng):
        edge = eng.relation("edge")
        out = eng.relation("out", index_flag=False)
        eng.load(edge, e)
        eng.load(out, None)
        lie = eng.lie()
        lie.add_relations(edge, True)
        lie.add_relations(out, False)
        lie.add_join(edge, FULL, edge, FULL, out, (INNER(1), OUTER(1)), pred=(kind, 0, 1))
        it = lie.fixpoint()
        return it, out.size(), out.digest(), out.rows().tolist()

    with Engine("oracle") as o:
        want = prog(o)
    with Engine("oracle_bitset") as b:
        got = prog(b)
    assert got == want


def test_bitset_oracle_refuses_what_it_cannot_hold():
    with Engine("oracle_bitset") as b:
        with pytest.raises(GdlError):
            b.relation("p3", arity=3)
        r = b.relation("r")
        with pytest.raises(GdlError):
            b.load(r, np.array([[1 << 15, 0]], dtype=np.uint64))
        b.load(r, np.array([[1, 2]], dtype=np.uint64))
        lie = b.lie()
        with pytest.raises(GdlError):
            lie.add_join(r, FULL, r, DELTA, r, (INNER(1), OUTER(1) | (1 << 8)))


def test_bitset_oracle_domain_grows_between_loads():
    """A later load with larger ids re-lays the matrices out."""
    with Engine("oracle_bitset") as b, Engine("oracle") as o:
        out = []
        for eng in (b, o):
            x = eng.relation("x")
            y = eng.relation("y")
            eng.load(x, np.array([[1, 2], [2, 3]], dtype=np.uint64))
            eng.load(y, np.array([[3, 9000], [2, 7000]], dtype=np.uint64))
            lie = eng.lie()
            lie.add_relations(y, True)
            lie.add_relations(x, False)
            lie.add_join(y, FULL, x, DELTA, x, (OUTER(0), INNER(1)))
            lie.fixpoint()
            out.append((x.rows().tolist(), x.digest(), y.rows(NEWT).tolist()))
        assert out[0] == out[1]
