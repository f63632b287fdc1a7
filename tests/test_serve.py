"""Serving loop (serve.py): requests that arrive while others are on the
GPU are batched with continuous admission; every request's result (size,
digest of its sorted tuples, loop passes) is the same in the mix as when
it runs alone through the plain engine."""
import copy
import types

import pytest

import batch as B
import serve as S
from gdlog_b200 import Engine


def small_stream(n=40, seed=3):
    return S.make_stream(n, rate=2000.0, seed=seed, min_scale=5, max_scale=7, l_range=(3, 16),
                         w_range=(3, 16))


def test_stream_shape_and_estimates():
    reqs = S.make_stream(200, rate=200.0, seed=1, min_scale=5, max_scale=7, l_range=(3, 9),
                         w_range=(3, 9))
    kinds = [r.kind for r in reqs]
    assert 0.55 < kinds.count("tc") / len(kinds) < 0.85
    arr = [r.arrival for r in reqs]
    assert arr == sorted(arr) and 0.5 < arr[-1] < 2.0  # ~200 requests at 200/s
    assert all(r.est_bytes > 0 and r.est_tuples > 0 for r in reqs)


def test_take_respects_the_tuple_cap():
    """A batch's summed first-join candidates stay within the cap (its first
    request is always admitted, so one query can still run alone)."""
    reqs = small_stream(30)
    cap = max(r.est_tuples for r in reqs) * 2
    srv = S.Server(slots=1, budget_bytes=1 << 40, max_batch=64, tuple_cap=cap)
    srv.queue.extend(reqs)
    while srv.queue:
        batch = srv._take()
        assert batch and (len(batch) == 1 or sum(r.est_tuples for r in batch) <= cap)


def test_take_batches_one_kind_within_budget():
    reqs = small_stream(20)
    srv = S.Server(slots=1, budget_bytes=1 << 40, max_batch=5)
    srv.queue.extend(reqs)
    first = srv._take()
    assert len(first) <= 5 and len({r.kind for r in first}) == 1
    assert first[0] is reqs[0]
    assert len(srv.queue) == len(reqs) - len(first)


def test_large_queries_are_taken_alone():
    """A query on plain_min_nodes nodes or more, of either program, is served
    alone (plain engine); no batch holds one with other queries."""
    reqs = S.make_stream(60, rate=2000.0, seed=4, min_scale=5, max_scale=8, l_range=(3, 16),
                         w_range=(3, 16))
    lim = 1 << 7
    assert any(r.kind == "sg" and r.nodes >= lim for r in reqs)
    assert any(r.kind == "tc" and r.nodes >= lim for r in reqs)
    srv = S.Server(slots=1, budget_bytes=1 << 40, max_batch=64, plain_min_nodes=lim)
    srv.queue.extend(reqs)
    sizes = []
    while srv.queue:
        batch = srv._take()
        big = [r for r in batch if r.nodes >= lim]
        assert not big or len(batch) == 1
        sizes.append(len(batch))
    assert max(sizes) > 1


def test_single_query_batches_run_on_the_plain_engine(monkeypatch):
    """A batch of one runs through the plain engine (faster than a batch of
    one in the block-diagonal layout); larger batches run batched."""
    calls = []

    def plain(eng, prog, instances):
        calls.append(("plain", len(instances)))
        return types.SimpleNamespace(results=[None] * len(instances))

    def batched(eng, prog, instances, node_counts=None):
        calls.append(("batched", len(instances)))
        return types.SimpleNamespace(results=[None] * len(instances))

    monkeypatch.setattr(B, "run_plain_loop", plain)
    monkeypatch.setattr(B, "run_batched", batched)
    reqs = small_stream(6, seed=2)
    srv = S.Server(slots=1)
    srv._run(None, S.PROGRAMS["tc"], reqs[:1])
    srv._run(None, S.PROGRAMS["tc"], reqs[:3])
    assert calls == [("plain", 1), ("batched", 3)]


def test_count_pass_estimate_matches_degrees_on_the_oracle():
    """The admission estimate from the first join's count pass (here the
    oracle's restatement of get_join_result_size) equals the host's
    degree-based cross-check, for transitive-closure and same-generation
    queries."""
    reqs = S.make_stream(24, rate=2000.0, seed=11, min_scale=5, max_scale=8, l_range=(3, 12),
                         w_range=(3, 12))
    assert {r.kind for r in reqs} == {"tc", "sg"}
    with Engine("oracle") as o:
        for r in reqs:
            assert S.device_estimate(o, r) == S.hbm_estimate(r), r.id


def test_join_count_edge_cases_on_the_oracle():
    """Empty sides count zero (a loaded relation's DELTA is empty until a
    LIE starts, src/lie.cu:49-59); keys present on one side only add
    nothing."""
    import numpy as np
    from gdlog_b200 import DELTA, FULL
    with Engine("oracle") as o:
        a = o.relation("a")
        b = o.relation("b")
        empty = o.relation("empty")
        o.load(a, np.array([[1, 2], [1, 3], [2, 5], [7, 7]], dtype=np.uint64))
        o.load(b, np.array([[1, 9], [2, 8], [2, 9], [4, 4]], dtype=np.uint64))
        o.load(empty, None)
        assert o.join_count(a, FULL, b, FULL) == 2 * 1 + 1 * 2  # keys 1 and 2
        assert o.join_count(b, FULL, a, FULL) == 1 * 2 + 2 * 1
        assert o.join_count(a, DELTA, b, FULL) == 0
        assert o.join_count(b, FULL, a, DELTA) == 0
        assert o.join_count(empty, FULL, a, FULL) == 0
        assert o.join_count(a, FULL, empty, FULL) == 0


@pytest.mark.gpu
def test_device_count_pass_matches_oracle_and_degrees():
    """gdl_join_count on the GPU (k_join_count over the loaded relations)
    gives the oracle's count and the host's degree estimate."""
    reqs = S.make_stream(24, rate=2000.0, seed=11, min_scale=6, max_scale=12, l_range=(3, 40),
                         w_range=(3, 40))
    with Engine("gpu") as g, Engine("oracle") as o:
        for r in reqs:
            want = S.hbm_estimate(r)
            assert S.device_estimate(g, r) == want, r.id
            assert S.device_estimate(o, r) == want, r.id


@pytest.mark.gpu
def test_device_join_count_edge_cases():
    import numpy as np
    from gdlog_b200 import DELTA, FULL, GdlError
    with Engine("gpu") as g:
        a = g.relation("a")
        b = g.relation("b")
        empty = g.relation("empty")
        noidx = g.relation("noidx", index_flag=False)
        g.load(a, np.array([[1, 2], [1, 3], [2, 5], [7, 7]], dtype=np.uint64))
        g.load(b, np.array([[1, 9], [2, 8], [2, 9], [4, 4]], dtype=np.uint64))
        g.load(empty, None)
        g.load(noidx, np.array([[1, 1]], dtype=np.uint64))
        assert g.join_count(a, FULL, b, FULL) == 4
        assert g.join_count(b, FULL, a, FULL) == 4
        assert g.join_count(empty, FULL, a, FULL) == 0
        assert g.join_count(a, FULL, empty, FULL) == 0
        assert g.join_count(b, FULL, a, DELTA) == 0
        assert g.size(a) == 4 and g.size(b) == 4  # nothing changed
        with pytest.raises(GdlError):
            g.join_count(noidx, FULL, a, FULL)
        with pytest.raises(GdlError):
            g.join_count(a, 2, b, FULL)  # NEWT is not a count-pass version


@pytest.mark.gpu
@pytest.mark.parametrize("plain_min_nodes", [0, 1 << 6])
def test_results_same_alone_and_in_the_mix(plain_min_nodes):
    reqs = small_stream()
    mixed = copy.deepcopy(reqs)
    stats = S.Server(slots=2, budget_bytes=1 << 30, max_batch=16,
                     plain_min_nodes=plain_min_nodes).serve(mixed)
    assert stats["requests"] == len(reqs)
    assert stats["mean_batch"] > 1.0  # arrivals overlap, so queries were batched
    with Engine("gpu") as g:
        for r, m in zip(reqs, mixed):
            alone = B.run_plain_loop(g, S.PROGRAMS[r.kind], [r.inputs]).results[0]
            assert (m.result.sizes, m.result.digests, m.result.iterations) == \
                (alone.sizes, alone.digests, alone.iterations), r.id


@pytest.mark.gpu
def test_plain_server_serves_everything():
    reqs = small_stream(12, seed=5)
    stats = S.Server(slots=1, batched=False).serve(reqs)
    assert stats["requests"] == 12 and stats["batches"] == 12
    assert all(r.result is not None for r in reqs)


@pytest.mark.gpu
def test_refused_batch_is_split_and_served(monkeypatch):
    """A batch the engine refuses for its size is run again in halves; every
    query still gets the result it gets alone."""
    import gdlog_b200 as G
    reqs = small_stream(10, seed=9)
    real = B.run_batched
    calls = []

    def picky(eng, prog, instances, node_counts=None):
        calls.append(len(instances))
        if len(instances) > 2:  # stand-in for the engine's list limit
            raise G.GdlError(4, "relation exceeds the tuple limit")
        return real(eng, prog, instances, node_counts=node_counts)

    monkeypatch.setattr(S.B, "run_batched", picky)
    srv = S.Server(slots=1, budget_bytes=1 << 40, max_batch=8)
    srv.queue.extend(reqs)
    srv.done = True
    srv._work(0.0)
    assert srv.splits > 0 and all(r.result is not None for r in reqs)
    monkeypatch.setattr(S.B, "run_batched", real)
    with Engine("gpu") as g:
        for r in reqs:
            alone = B.run_plain_loop(g, S.PROGRAMS[r.kind], [r.inputs]).results[0]
            assert (r.result.sizes, r.result.digests, r.result.iterations) == \
                (alone.sizes, alone.digests, alone.iterations), r.id
