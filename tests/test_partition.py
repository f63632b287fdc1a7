"""Partitioned fixpoint (partition.py): transitive closure and same
generation with their relations hash-partitioned over ranks and
all-to-all exchanges of new tuples per pass.  On CPU: 2 and 3 gloo ranks,
each with the oracle as its engine, against one oracle run (the same result
and the same loop-pass counts).  On a GPU: one rank over the CUDA engine."""
import json
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import partition as PT
import programs as P
import workloads as W
from gdlog_b200 import Engine

CASES = {
    "grid_10": lambda: W.grid_edges(10, 10),
    "dag_L12_W10": lambda: W.layered_dag(12, 10, 1),
    "rmat_s7": lambda: W.rmat_edges(7, 300, seed=3),
}


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, case, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                           world_size=world)
    try:
        with Engine("oracle") as eng:
            res = PT.partitioned_tc(eng, CASES[case](), rank, world)
        rows = PT.gather_rows(res.full, world)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"passes": res.passes, "n": len(res.full), "rows": rows.tolist(),
                       "per_pass": res.per_pass_new}, f)
    finally:
        dist.destroy_process_group()


def single(case):
    with Engine("oracle") as o:
        r = P.tc(o, CASES[case]())
        rows = r.output.rows()
        return r.iterations["tc"], rows[np.lexsort((rows[:, 1], rows[:, 0]))].tolist()


@pytest.mark.parametrize("case,world", [(c, 2) for c in sorted(CASES)] + [("grid_10", 3)])
def test_partitioned_tc_equals_single(case, world, tmp_path):
    mp.spawn(_rank, args=(world, free_port(), case, str(tmp_path)), nprocs=world, join=True)
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    iters, rows = single(case)
    for o in outs:
        assert o["passes"] == iters
        assert o["rows"] == rows
    assert sum(o["n"] for o in outs) == len(rows)  # disjoint partitions


SG_CASES = {
    "rmat_s7": lambda: W.rmat_edges(7, 300, seed=3),
    "rmat_s8": lambda: W.rmat_edges(8, 600, seed=1),
    "dag_L8_W6": lambda: W.layered_dag(8, 6, 2),
}


def _rank_sg(rank, world, port, case, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        with Engine("oracle") as eng:
            res = PT.partitioned_sg(eng, SG_CASES[case](), rank, world)
        rows = PT.gather_rows(res.full, world)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"init": res.init_passes, "sg": res.passes, "n": len(res.full),
                       "rows": rows.tolist()}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world", [(c, 2) for c in sorted(SG_CASES)] + [("rmat_s8", 3)])
def test_partitioned_sg_equals_single(case, world, tmp_path):
    mp.spawn(_rank_sg, args=(world, free_port(), case, str(tmp_path)), nprocs=world, join=True)
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    with Engine("oracle") as o:
        r = P.sg(o, SG_CASES[case]())
        want = r.output.rows()
        want = want[np.lexsort((want[:, 1], want[:, 0]))].tolist()
        iters = r.iterations
    for o in outs:
        assert (o["init"], o["sg"]) == (iters["init"], iters["sg"])
        assert o["rows"] == want
    assert sum(o["n"] for o in outs) == len(want)


def test_owner_and_route_shapes():
    ids = np.array([0, 1, 2, 3, 7, 10])
    assert PT.owner(ids, 3).tolist() == [0, 1, 2, 0, 1, 1]
    rows = np.array([[5, 1], [2, 3], [1 << 20, 7], [(1 << 32) - 1, (1 << 31) + 5]],
                    dtype=np.uint64)
    assert (PT._unpack(PT._pack(rows)) == rows).all()
    assert PT._unpack(PT._pack(np.zeros((0, 2), np.uint64))).shape == (0, 2)
    tri = np.array([[7, (1 << 32) - 1, 3], [0, 1, 2]], dtype=np.uint64)
    assert (PT._rows_of(PT._keys_of(tri), 3) == tri).all()
    assert (PT._rows_of(PT._keys_of(rows), 2) == rows).all()


@pytest.mark.gpu
def test_partitioned_tc_one_rank_on_the_gpu():
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{free_port()}", rank=0,
                            world_size=1)
    try:
        e = W.grid_edges(24, 24)
        with Engine("gpu") as g:
            res = PT.partitioned_tc(g, e, 0, 1)
            full = res.full[np.lexsort((res.full[:, 1], res.full[:, 0]))]
        with Engine("gpu") as g:
            r = P.tc(g, e, sync=g.sync)
            want = r.output.rows()
            assert res.passes == r.iterations["tc"]
        assert full.tolist() == want[np.lexsort((want[:, 1], want[:, 0]))].tolist()
    finally:
        dist.destroy_process_group()


def _rank_gpu(rank, world, port, prog, case, out_dir):
    """A rank of a partitioned fixpoint over the CUDA engine with the
    exchange kept on the device (DeviceExchange); the ranks share one GPU
    and synchronise only through gloo collectives on the host."""
    import torch
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        with Engine("gpu") as eng:
            if prog == "tc":
                res = PT.partitioned_tc(eng, CASES[case](), rank, world)
                passes = {"tc": res.passes}
            else:
                res = PT.partitioned_sg(eng, SG_CASES[case](), rank, world)
                passes = {"init": res.init_passes, "sg": res.passes}
        rows = PT.gather_rows(res.full, world)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"passes": passes, "n": len(res.full), "rows": rows.tolist()}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("prog,case", [("tc", "grid_10"), ("tc", "rmat_s7"), ("sg", "rmat_s8"),
                                       ("sg", "dag_L8_W6")])
def test_device_resident_exchange_two_ranks(prog, case, tmp_path):
    """Two ranks, each over the CUDA engine with its candidates exported,
    grouped by owner, exchanged and reloaded in device memory, give the
    single-engine result and loop-pass counts."""
    world = 2
    mp.spawn(_rank_gpu, args=(world, free_port(), prog, case, str(tmp_path)), nprocs=world,
             join=True)
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    with Engine("oracle") as o:
        if prog == "tc":
            r = P.tc(o, CASES[case]())
        else:
            r = P.sg(o, SG_CASES[case]())
        want = r.output.rows()
        want = want[np.lexsort((want[:, 1], want[:, 0]))].tolist()
        iters = dict(r.iterations)
    for o in outs:
        assert o["passes"] == iters
        assert o["rows"] == want
    assert sum(o["n"] for o in outs) == len(want)


@pytest.mark.gpu
def test_partition_rows_groups_by_owner():
    """gdl_partition_rows: each row lands in its owner's block, block sizes
    are the owners' counts, nothing is lost or repeated."""
    import torch
    rng = np.random.default_rng(5)
    rows = np.stack([rng.integers(0, 1 << 32, 5000, dtype=np.uint64),
                     rng.integers(0, 1 << 20, 5000, dtype=np.uint64)], axis=1)
    with Engine("gpu") as g:
        src = torch.from_numpy(rows.view(np.int64)).cuda()
        out = torch.empty_like(src)
        for col, world in ((0, 3), (1, 7), (0, 1)):
            counts = g.partition_rows(src.data_ptr(), len(rows), col, world, out.data_ptr())
            got = out.cpu().numpy().view(np.uint64)
            assert counts == np.bincount((rows[:, col] % world).astype(np.int64),
                                         minlength=world).tolist()
            at = 0
            for d, c in enumerate(counts):
                block = got[at:at + c]
                assert (block[:, col] % world == d).all()
                at += c
            key = lambda a: np.lexsort((a[:, 1], a[:, 0]))  # noqa: E731
            assert (got[key(got)] == rows[key(rows)]).all()
        assert g.partition_rows(0, 0, 0, 4, 0) == [0, 0, 0, 0]
