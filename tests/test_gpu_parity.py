"""GPU parity: the CUDA engine, called through its C-ABI, against the oracle.

Bit-exact on every count: result sizes, loop-pass counts, the per-iteration
(dedup, delta, full) log of src/lie.cu:193-197 and the order-sensitive
digest of the sorted result tuples.  Small workloads are compared with the
committed golden fixtures; the full-size ones (64x64 grid TC, R-MAT scale
14 SG) with their golden digests and with size-independent properties
(sortedness, uniqueness) of the exported rows.
"""
import json
import os

import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import (DELTA, FULL, INNER, NEWT, OUTER, PRED_GT, PRED_LT, PRED_NE, SRC, Engine,
                        GdlError)
from test_oracle import GOLDEN, SMALL, build_workload

pytestmark = pytest.mark.gpu

# Both deduplication paths of the engine: radix sort + merge-path merge, and
# bitmaps over the key domain (every workload here has a small domain, so
# "dense" is what the engine picks by itself); bitmaps with every eligible
# join in the pull form (gathered by output row) or every join in the push
# form, or every eligible join gathered along its static inner's in-edges
# (row-gather form); bitmaps with dirty maps at every size (scans of listed dirty
# chunks), bitmaps with push joins as count + materialise passes instead of
# one probe-and-expand pass, and bitmaps whose push joins combine a warp's
# bits per word before the reduction.
MODES = ["sort", "dense", "dense_pull", "dense_push", "dense_dirty", "dense_2pass", "dense_agg",
         "dense_rows"]


def summarize(r):
    return {
        "sizes": {k: v.size() for k, v in r.relations.items()},
        "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
        "iterations": r.iterations,
        "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
    }


def run_both(prog, *args, mode="dense"):
    with Engine("gpu", dedup=mode) as g:
        got = summarize(prog(g, *args, sync=g.sync))
    with Engine("oracle") as o:
        want = summarize(prog(o, *args))
    return got, want


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", SMALL)
def test_small_workloads_match_golden(name, mode):
    prog, args = build_workload(name)
    with Engine("gpu", dedup=mode) as g:
        got = summarize(prog(g, *args, sync=g.sync))
    want = GOLDEN["workloads"][name]
    assert got["sizes"] == want["sizes"]
    assert got["iterations"] == want["iterations"]
    assert got["digests"] == want["digests"]
    assert got["traces"] == want["traces"]


@pytest.mark.parametrize("mode", MODES)
def test_grid_tc_64x64(mode):
    want = GOLDEN["workloads"]["tc_grid_64x64"]
    with Engine("gpu", dedup=mode) as g:
        r = P.tc(g, W.grid_edges(64, 64), sync=g.sync)
        assert r.output.size() == 4322304
        assert r.iterations["tc"] == 126
        assert hex(r.output.digest()) == want["digests"]["path"]
        assert r.lies["tc"].trace().tolist() == want["traces"]["tc"]


@pytest.mark.parametrize("mode", MODES)
def test_sg_rmat_scale14_full_size(mode):
    want = GOLDEN["workloads"]["sg_rmat_s14_40000_s14"]
    with Engine("gpu", dedup=mode) as g:
        r = P.sg(g, W.rmat_edges(14, 40000, seed=14), sync=g.sync)
        assert r.output.size() == want["sizes"]["sg"]
        assert r.iterations == want["iterations"]
        assert hex(r.output.digest()) == want["digests"]["sg"]
        rows = r.output.rows()
        key = (rows[:, 0] << np.uint64(32)) | rows[:, 1]
        assert (np.diff(key.astype(np.int64)) > 0).all()  # sorted, unique
        assert rows.max() < 2**14


@pytest.mark.parametrize("mode", MODES)
def test_graph_and_stream_paths_agree(mode):
    e = W.layered_dag(20, 12, 7)
    os.environ["GDLOG_NO_GRAPH"] = "1"
    try:
        with Engine("gpu", dedup=mode) as g:
            a = summarize(P.tc(g, e, sync=g.sync))
    finally:
        del os.environ["GDLOG_NO_GRAPH"]
    with Engine("gpu", dedup=mode) as g:
        b = summarize(P.tc(g, e, sync=g.sync))
    assert a == b


@pytest.mark.parametrize("mode", MODES)
def test_duplicate_and_unsorted_input(mode):
    e = W.layered_dag(10, 9, 3)
    noisy = np.concatenate([e[::-1], e[: len(e) // 2]])
    got, want = run_both(P.tc, noisy, mode=mode)
    assert got == want


@pytest.mark.parametrize("mode", MODES)
def test_empty_relation(mode):
    e = np.zeros((0, 2), dtype=np.uint64)
    got, want = run_both(P.tc, e, mode=mode)
    assert got == want
    assert got["sizes"]["path"] == 0


def test_large_ids_hashed_index():
    """Column values above the identity-index range use the hashed index."""
    e = W.layered_dag(12, 10, 5) * np.uint64(40503) + np.uint64(3_000_000_000)
    got, want = run_both(P.tc, e)
    assert got == want


def test_values_above_32_bits_rejected():
    with Engine("gpu") as g:
        r = g.relation("x")
        with pytest.raises(GdlError):
            g.load(r, np.array([[1 << 33, 1]], dtype=np.uint64))


@pytest.mark.parametrize("mode", MODES)
def test_max_iteration_cap(mode):
    e = W.grid_edges(12, 12)
    for cap in (0, 1, 5):
        res = []
        for kind in ("gpu", "oracle"):
            with Engine(kind, dedup=mode if kind == "gpu" else None) as eng:
                path = eng.relation("path", index_flag=False)
                edge = eng.relation("edge")
                eng.load(path, e)
                eng.load(edge, W.reverse(e))
                lie = eng.lie()
                lie.set_reload_full(False)
                lie.add_relations(edge, True)
                lie.add_relations(path, False)
                lie.add_join(edge, FULL, path, DELTA, path, P.REORDER_PATH)
                lie.max_iteration = cap
                it = lie.fixpoint()
                res.append((it, path.size(), path.digest(), lie.trace().tolist()))
        assert res[0] == res[1], cap


def empty_inner_program(eng):
    """A join whose inner is empty zeroes the outer's count
    (src/join.cu:38-45); a Copy from an empty source zeroes the dest NEWT
    (src/copy.cu:24-27)."""
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


@pytest.mark.parametrize("mode", MODES)
def test_empty_inner_quirk(mode):
    with Engine("gpu", dedup=mode) as g:
        got = empty_inner_program(g)
    with Engine("oracle") as o:
        want = empty_inner_program(o)
    assert got == want


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", [PRED_NE, PRED_LT, PRED_GT])
def test_predicates(kind, mode):
    e = W.rmat_edges(7, 300, seed=9)

    def prog(eng, sync=None):
        edge = eng.relation("edge")
        out = eng.relation("out", index_flag=False)
        eng.load(edge, e)
        eng.load(out, None)
        lie = eng.lie()
        lie.add_relations(edge, True)
        lie.add_relations(out, False)
        lie.add_join(edge, FULL, edge, FULL, out, (INNER(1), OUTER(1)), pred=(kind, 0, 1))
        it = lie.fixpoint()
        return it, out.size(), out.digest()

    with Engine("gpu", dedup=mode) as g:
        got = prog(g)
    with Engine("oracle") as o:
        want = prog(o)
    assert got == want


def test_relation_export_roundtrip():
    rows = np.array([[7, 1], [0, 9], [7, 0], [0, 9]], dtype=np.uint64)
    with Engine("gpu") as g:
        r = g.relation("x")
        g.load(r, rows)
        assert r.size() == 3
        assert r.rows().tolist() == [[0, 9], [7, 0], [7, 1]]


@pytest.mark.parametrize("mode", MODES)
def test_repeated_fixpoints_on_one_engine(mode):
    """Engine state (scratch buffers, index epochs, look-back generations)
    carries over correctly from one program to the next."""
    with Engine("gpu", dedup=mode) as g:
        outs = []
        for seed in (1, 2, 3):
            prog, args = build_workload(f"sg_rmat_s8_600_s{seed}")
            outs.append(summarize(prog(g, *args, sync=g.sync)))
    for seed, got in zip((1, 2, 3), outs):
        want = GOLDEN["workloads"][f"sg_rmat_s8_600_s{seed}"]
        assert got["sizes"] == want["sizes"] and got["digests"] == want["digests"]


def test_modes_agree_on_cspa_with_clear():
    """Sort and dense paths give identical CSPA results on one engine that
    is cleared between programs (scratch and bitmaps are reused)."""
    assign, deref = W.cspa_facts(200, 400, 150, seed=8)
    out = []
    with Engine("gpu") as g:
        for mode, dirty in (("sort", 24), ("dense", 24), ("dense", 11), ("sort", 24)):
            g.clear()
            g.set_tuning(dedup=mode, dirty_min_log2_words=dirty)
            out.append(summarize(P.cspa(g, assign, deref, sync=g.sync)))
    with Engine("oracle") as o:
        want = summarize(P.cspa(o, assign, deref))
    assert out[0] == out[1] == out[2] == out[3] == want


@pytest.mark.parametrize("mode", ["dense", "sort"])
def test_ids_up_to_2_16_match_oracle(mode):
    """Ids above 2^15 (a 2^32-bit key domain: 512 MB bitmaps, rows of one
    scan tile): both paths still match the oracle."""
    e = W.rmat_edges(16, 3000, seed=21)
    assert int(e.max()) >= 1 << 15
    with Engine("gpu", dedup=mode) as g:
        got = summarize(P.sg(g, e, sync=g.sync))
    with Engine("oracle") as o:
        want = summarize(P.sg(o, e))
    assert got == want


def dag_closure_size(L, Wd, seed):
    """|TC| of a layered DAG from reachability bitsets, layer by layer from
    the last one (independent of both engines)."""
    e = W.layered_dag(L, Wd, seed).astype(np.int64)
    n = L * Wd
    words = (n + 63) // 64
    reach = np.zeros((n, words), dtype=np.uint64)
    succ = [[] for _ in range(n)]
    for a, b in e.tolist():
        succ[a].append(b)
    for x in range(n - 1, -1, -1):
        for y in succ[x]:
            reach[x] |= reach[y]
            reach[x, y // 64] |= np.uint64(1) << np.uint64(y % 64)
    return int(np.bitwise_count(reach).sum())


def test_closure_beyond_the_list_limit_stays_a_bitmap():
    """A closure of more than 2^30 pairs (60,000 nodes) cannot be a list:
    FULL stays the bitmap, whose size and digest are still readable and
    whose rows are refused with a status."""
    L, Wd, seed = 200, 300, 5
    e = W.layered_dag(L, Wd, seed)
    with Engine("gpu") as g:
        r = P.tc(g, e, sync=g.sync)
        path = r.output
        n = path.size()
        d1 = path.digest()
        assert n > (1 << 30)
        with pytest.raises(GdlError):
            path.rows()
        assert path.digest() == d1
    assert n == dag_closure_size(L, Wd, seed)
