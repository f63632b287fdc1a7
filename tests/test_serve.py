"""Serving loop (serve.py): requests that arrive while others are on the
GPU are batched with continuous admission; every request's result (size,
digest of its sorted tuples, loop passes) is the same in the mix as when
it runs alone through the plain engine."""
import copy

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
    assert all(r.est_bytes > 0 for r in reqs)


def test_take_batches_one_kind_within_budget():
    reqs = small_stream(20)
    srv = S.Server(slots=1, budget_bytes=1 << 40, max_batch=5)
    srv.queue.extend(reqs)
    first = srv._take()
    assert len(first) <= 5 and len({r.kind for r in first}) == 1
    assert first[0] is reqs[0]
    assert len(srv.queue) == len(reqs) - len(first)


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix():
    reqs = small_stream()
    mixed = copy.deepcopy(reqs)
    stats = S.Server(slots=2, budget_bytes=1 << 30, max_batch=16).serve(mixed)
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
