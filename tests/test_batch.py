"""Batched fixpoints (batch.py, gdl_engine_set_instances): every instance's
result -- size, digest of its sorted tuples in local ids, and the loop-pass
count it would have taken alone -- is bit-exact against the plain engine
run instance by instance, and against the oracle."""
import numpy as np
import pytest

import batch as B
import programs as P
import workloads as W
from gdlog_b200 import Engine


def dag_instances(n, seed, l_range=(2, 10), w_range=(2, 9)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = int(rng.integers(*l_range))
        Wd = int(rng.integers(*w_range))
        out.append((W.layered_dag(L, Wd, seed * 1000 + i),))
    return out


def sg_instances(n, seed):
    rng = np.random.default_rng(seed)
    return [(W.rmat_edges(int(rng.integers(4, 7)), int(rng.integers(20, 90)), seed=seed * 100 + i),)
            for i in range(n)]


def cspa_instances(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        v = int(rng.integers(8, 40))
        out.append(W.cspa_facts(v, 2 * v, v, seed=seed * 100 + i))
    return out


def as_tuples(run):
    return [(r.sizes, r.digests, r.iterations) for r in run.results]


def test_globalize_moves_ids_into_instance_ranges():
    a = np.array([[0, 1], [1, 2]], dtype=np.uint64)
    b = np.array([[0, 0]], dtype=np.uint64)
    (g,) = B.globalize([(a,), (b,)], shift=3)
    assert g.tolist() == [[0, 1], [1, 2], [8, 8]]
    assert B.node_count((a,)) == 3 and B.node_count((np.zeros((0, 2)),)) == 1


def test_batched_oracle_loop_matches_itself():
    inst = dag_instances(4, 1)
    with Engine("oracle") as o:
        r1 = B.run_plain_loop(o, P.tc, inst)
        r2 = B.run_plain_loop(o, P.tc, inst)
    assert as_tuples(r1) == as_tuples(r2)


@pytest.mark.gpu
@pytest.mark.parametrize("seed,dirty,agg", [(1, 24, 1), (2, 11, 1), (3, 11, 2)])
def test_batched_tc_matches_plain_and_oracle(seed, dirty, agg):
    inst = dag_instances(12, seed)
    inst.append((np.zeros((0, 2), dtype=np.uint64),))  # an instance without edges
    with Engine("gpu") as g:
        g.set_tuning(dirty_min_log2_words=dirty, join_aggregate=agg)
        batched = B.run_batched(g, P.tc, inst)
        plain = B.run_plain_loop(g, P.tc, inst)
    with Engine("oracle") as o:
        oracle = B.run_plain_loop(o, P.tc, inst)
    assert as_tuples(batched) == as_tuples(plain) == as_tuples(oracle)


@pytest.mark.gpu
def test_batched_sg_matches_oracle():
    inst = sg_instances(8, 3)
    with Engine("gpu") as g:
        g.set_tuning(dirty_min_log2_words=11)
        batched = B.run_batched(g, P.sg, inst)
    with Engine("oracle") as o:
        oracle = B.run_plain_loop(o, P.sg, inst)
    assert as_tuples(batched) == as_tuples(oracle)


@pytest.mark.gpu
def test_batched_cspa_matches_oracle():
    inst = cspa_instances(6, 4)
    with Engine("gpu") as g:
        g.set_tuning(dirty_min_log2_words=11)
        batched = B.run_batched(g, P.cspa, inst)
    with Engine("oracle") as o:
        oracle = B.run_plain_loop(o, P.cspa, inst)
    assert as_tuples(batched) == as_tuples(oracle)


@pytest.mark.gpu
def test_batched_large_instances_keep_full_as_bitmap():
    """Uneven instances up to thousands of nodes, as in the 384-DAG
    workload; per-instance results still match the plain engine."""
    inst = [(W.layered_dag(L, Wd, 77 + i),) for i, (L, Wd) in
            enumerate([(40, 64), (8, 16), (100, 30), (3, 250), (60, 100)])]
    with Engine("gpu") as g:
        batched = B.run_batched(g, P.tc, inst)
        plain = B.run_plain_loop(g, P.tc, inst)
    assert as_tuples(batched) == as_tuples(plain)


def test_shard_instances_partitions_and_balances():
    costs = [float(c) for c in np.random.default_rng(5).integers(1, 1000, size=97)]
    for world in (1, 2, 3, 8):
        parts = [B.shard_instances(costs, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)


def _shard_worker(rank, world, port, costs, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    mine = B.shard_instances(costs, world, rank)
    out = [None] * world
    dist.all_gather_object(out, mine)
    if rank == 0:
        q.put(out)
    dist.destroy_process_group()


def test_shard_instances_agree_across_gloo_ranks():
    """Every rank computes the same partition without exchanging work."""
    import multiprocessing as mp
    import socket

    costs = [float(c) for c in np.random.default_rng(9).integers(1, 500, size=40)]
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
    assert sorted(parts[0] + parts[1]) == list(range(40))
    assert not set(parts[0]) & set(parts[1])
    assert parts == [B.shard_instances(costs, 2, r) for r in range(2)]


@pytest.mark.gpu
def test_batched_cspa_long_runs_match_oracle():
    """CSPA instances large enough for runs longer than a bitmap row, so the
    joins OR whole rows of the inner's FULL bitmap in the block-diagonal
    layout; every instance still matches the oracle."""
    inst = [W.cspa_facts(v, 2 * v, 3 * v // 4, seed=40 + v) for v in (260, 300, 200)]
    with Engine("gpu") as g:
        batched = B.run_batched(g, P.cspa, inst)
    with Engine("oracle") as o:
        oracle = B.run_plain_loop(o, P.cspa, inst)
    assert as_tuples(batched) == as_tuples(oracle)
