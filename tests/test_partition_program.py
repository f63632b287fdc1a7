"""Any Datalog program of the front end, partitioned (partition.py:
partitioned_program): 2 and 3 gloo ranks, each with the oracle as its
engine, against datalog.run on one oracle engine — the same rows for every
head predicate (the union of the partitions, which are disjoint) and the
same loop-pass count for every component."""
import json
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import datalog as D
import partition as PT
import workloads as W
from gdlog_b200 import Engine

TC = """
path(x, y) :- edge(x, y).
path(x, z) :- path(x, y), edge(y, z).
"""

TC_NONLINEAR = """
path(x, y) :- edge(x, y).
path(x, z) :- path(x, y), path(y, z).
"""

SG = """
sg(x, y) :- edge(p, x), edge(p, y), x != y.
sg(x, y) :- edge(a, x), sg(a, b), edge(b, y).
"""

CSPA = """
vf(y, y) :- assign(x, y).
vf(x, x) :- assign(x, y).
vf(x, y) :- assign(x, y).
ma(y, y) :- assign(x, y).
ma(x, x) :- assign(x, y).
vf(x, y) :- vf(x, z), vf(z, y).
va(x, y) :- vf(z, x), vf(z, y).
vf(x, y) :- assign(x, z), ma(z, y).
ma(x, w) :- deref(y, x), va(y, z), deref(z, w).
va(x, y) :- vf(z, x), ma(z, w), vf(w, y).
"""

PLEN = """
path(x, y, 1) :- edge(x, y).
path(x, y, l+1) :- edge(x, m), path(m, y, l).
"""

STRATA = """
sym(x, y) :- e(x, y).
sym(x, y) :- e(y, x).
reach(x, y) :- sym(x, y).
reach(x, z) :- reach(x, y), sym(y, z).
"""

EMPTY = """
p(x, y) :- e(x, y).
p(x, z) :- p(x, y), f(y, z).
q(x, y) :- f(x, y).
q(x, z) :- q(x, y), e(y, z).
"""


MIRROR_SEEDS = """
r(x, 0) :- e(x, y).
r(x, z) :- r(x, y), e(y, z).
"""


def _mirror_seeds():
    r = _u(W.rmat_edges(5, 20, seed=9))
    return {"e": _u(W.rmat_edges(5, 40, seed=2)), "r": r[r[:, 1] != 0]}


def _u(rows):
    return np.unique(np.asarray(rows, dtype=np.uint64), axis=0)


def _cspa():
    assign, deref = W.cspa_facts(120, 240, 90, seed=1)
    return {"assign": _u(assign), "deref": _u(deref)}


CASES = {
    "tc_grid_8": (TC, lambda: {"edge": _u(W.grid_edges(8, 8))}, None),
    "tc_rmat_s7": (TC, lambda: {"edge": _u(W.rmat_edges(7, 300, seed=5))}, None),
    "tc_nonlinear_rmat_s7": (TC_NONLINEAR, lambda: {"edge": _u(W.rmat_edges(7, 300, seed=5))},
                             None),
    "sg_rmat_s7": (SG, lambda: {"edge": _u(W.rmat_edges(7, 300, seed=3))}, None),
    "cspa_120": (CSPA, _cspa, None),
    "plen_rmat_s6": (PLEN, lambda: {"edge": _u(W.rmat_edges(6, 150, seed=6))}, {"path": 1}),
    "strata_rmat_s6": (STRATA, lambda: {"e": _u(W.rmat_edges(6, 60, seed=8))}, None),
    # an empty inner zeroes the outer's DELTA, a Copy from an empty input
    # clears its destination's NEWT (src/join.cu:38-45, src/copy.cu:24-27)
    "empty_inner": (EMPTY, lambda: {"e": _u(W.grid_edges(5, 5)),
                                    "f": np.zeros((0, 2), np.uint64)}, None),
    # every id a multiple of 6: at 2 and 3 ranks one rank owns every key
    "one_owner": (TC, lambda: {"edge": _u(W.grid_edges(6, 6)) * np.uint64(6)}, None),
    "mirror_seeds": (MIRROR_SEEDS, lambda: _mirror_seeds(), None),
}


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sorted(rows):
    return sorted(map(tuple, np.asarray(rows).tolist()))


def _rank(rank, world, port, case, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        text, inputs, deps = CASES[case]
        with Engine("oracle", max_arity=3) as eng:
            res = PT.partitioned_program(eng, text, inputs(), rank, world, deps=deps)
        out = {"iterations": res.iterations, "relations": res.relations, "rows": {}, "n": {}}
        for p, rows in sorted(res.full.items()):
            parts = [None] * world
            dist.all_gather_object(parts, np.asarray(rows, dtype=np.uint64))
            out["rows"][p] = [list(r) for r in _sorted(np.concatenate(parts))]
            out["n"][p] = len(rows)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world", [(c, 2) for c in sorted(CASES)] +
                         [("cspa_120", 3), ("sg_rmat_s7", 3), ("plen_rmat_s6", 3),
                          ("one_owner", 3)])
def test_partitioned_program_equals_single(case, world, tmp_path):
    mp.spawn(_rank, args=(world, free_port(), case, str(tmp_path)), nprocs=world, join=True)
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    text, inputs, deps = CASES[case]
    with Engine("oracle", max_arity=3) as o:
        r = D.run(o, text, inputs(), deps=deps)
        want = {p: [list(x) for x in _sorted(rel.rows() if rel.size() else [])]
                for p, rel in r.relations.items()}
        iters = dict(r.iterations)
    for o in outs:
        assert o["iterations"] == iters
        assert sorted(o["rows"]) == sorted(want)
        for p in want:
            assert o["rows"][p] == want[p], p
        # the engine's relation table holds every relation a rank uses
        assert o["relations"] <= 64
    for p in want:  # disjoint partitions
        assert sum(o["n"][p] for o in outs) == len(want[p])


def test_program_file_under_torchrun(tmp_path):
    """`datalog.py prog.dl` under torchrun (2 gloo ranks, the oracle as each
    rank's engine) writes the same sorted output file and prints the same
    sizes and loop-pass counts as a run on one engine."""
    import subprocess
    import sys
    prog = tmp_path / "cspa.dl"
    prog.write_text(".decl assign(a: number, b: number)\n.input assign\n"
                    ".decl deref(a: number, b: number)\n.input deref\n"
                    ".decl vf(a: number, b: number)\n.output vf\n.printsize vf\n"
                    ".decl ma(a: number, b: number)\n.printsize ma\n"
                    ".decl va(a: number, b: number)\n.output va\n.printsize assign\n" + CSPA)
    assign, deref = W.cspa_facts(100, 200, 80, seed=4)
    for name, rows in (("assign", assign), ("deref", deref)):
        with open(tmp_path / f"{name}.facts", "w") as f:
            for a, b in np.asarray(rows).tolist():
                f.write(f"{a}\t{b}\n")
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = os.path.join(here, "gdlog-multinode_b200", "datalog.py")
    common = [str(prog), "--facts", str(tmp_path), "--engine", "oracle"]
    one = subprocess.run([sys.executable, script, *common, "--out", str(tmp_path / "one")],
                         capture_output=True, text=True, check=True, timeout=300)
    two = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                          "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                          "--master-port", str(free_port()), script, *common,
                          "--out", str(tmp_path / "two")],
                         capture_output=True, text=True, check=True, timeout=300)
    a = json.loads(one.stdout.strip().splitlines()[-1])
    b = json.loads([ln for ln in two.stdout.strip().splitlines() if ln.startswith("{")][-1])
    assert b["ranks"] == 2
    assert (b["sizes"], b["iterations"]) == (a["sizes"], a["iterations"])
    for name in ("vf", "va"):
        assert (tmp_path / "two" / f"{name}.csv").read_text() == \
            (tmp_path / "one" / f"{name}.csv").read_text()



def test_mirror_holds_seeds_and_inputs():
    """A predicate with input rows and a number-headed rule, joined on its
    second column (a swapped mirror): the mirror starts from all its loaded
    rows.  Checked against a closure computed here; the partitioned run is
    the case mirror_seeds above."""
    inputs = _mirror_seeds()
    with Engine("oracle") as o:
        got = _sorted(D.run(o, MIRROR_SEEDS, inputs).relations["r"].rows())
    r = set(map(tuple, inputs["r"].tolist())) | {(x, 0) for x, _ in inputs["e"].tolist()}
    e = inputs["e"].tolist()
    while True:
        new = {(x, z) for (x, y) in r for (y2, z) in e if y2 == y} - r
        if not new:
            break
        r |= new
    assert got == sorted(r)


def _rank_fails(rank, world, port, out_dir):
    import time
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=5))
    t0 = time.time()
    status = "ok"
    try:
        with Engine("oracle") as eng:
            inputs = {"edge": _u(W.grid_edges(4, 4))}
            if rank == 1:  # this rank's program names an input nobody passed
                PT.partitioned_program(eng, TC + "q(x, y) :- missing(x, y).\n", inputs,
                                       rank, world)
            else:
                PT.partitioned_program(eng, TC, inputs, rank, world)
    except Exception as exc:  # noqa: BLE001 - the failure is the result
        status = type(exc).__name__
    with open(os.path.join(out_dir, f"f{rank}.json"), "w") as f:
        json.dump({"status": status, "seconds": time.time() - t0}, f)
    try:
        dist.destroy_process_group()
    except Exception:  # noqa: BLE001 - the group may already be broken
        pass


def test_a_failed_rank_ends_the_others(tmp_path):
    """A rank that fails before its first exchange (on the host: a program
    that names no given input) leaves the other rank's next collective
    with an error within the process group's timeout, not waiting."""
    d = str(tmp_path)
    mp.spawn(_rank_fails, args=(2, free_port(), d), nprocs=2, join=True)
    f0 = json.load(open(os.path.join(d, "f0.json")))
    f1 = json.load(open(os.path.join(d, "f1.json")))
    assert f1["status"] == "ValueError"
    assert f0["status"] != "ok" and f0["seconds"] < 60


def _rank_count(rank, world, port, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    calls = {"all_reduce": 0, "all_to_all_single": 0}
    for name in calls:
        real = getattr(dist, name)

        def counted(*a, _real=real, _name=name, **k):
            calls[_name] += 1
            return _real(*a, **k)
        setattr(dist, name, counted)
    try:
        with Engine("oracle") as eng:
            res = PT.partitioned_program(eng, TC, {"edge": _u(W.grid_edges(6, 6))}, rank, world)
        with open(os.path.join(out_dir, f"c{rank}.json"), "w") as f:
            json.dump({"passes": res.iterations["path"], **calls}, f)
    finally:
        dist.destroy_process_group()


def test_collectives_per_pass(tmp_path):
    """Transitive closure partitioned (path joined on its second column, so
    a swapped mirror of path is kept too): one exchange of the mirror's
    first rows and one all_reduce of sizes when the component starts, then
    per pass one exchange of the new rows of path and its mirror together
    (an all_to_all of counts and one of keys) and one all_reduce of the
    new-tuple counts.  The Copy and the join read FULL and DELTA, whose
    global sizes are tracked, and the ACopy needs none, so they reduce
    nothing."""
    mp.spawn(_rank_count, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        c = json.load(open(tmp_path / f"c{r}.json"))
        assert c["all_reduce"] == 1 + c["passes"]
        assert c["all_to_all_single"] == 2 + 2 * c["passes"]


def _rank_gpu(rank, world, port, case, out_dir):
    """One rank with the CUDA engine.  The ranks share one GPU; their only
    connection is the gloo collectives on the host (no kernel waits on
    another rank's)."""
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        text, inputs, deps = CASES[case]
        with Engine("gpu", device=0) as eng:
            res = PT.partitioned_program(eng, text, inputs(), rank, world, deps=deps)
            out = {"iterations": res.iterations, "relations": res.relations, "rows": {},
                   "n": {}}
            for p, rows in sorted(res.full.items()):
                parts = [None] * world
                dist.all_gather_object(parts, np.asarray(rows, dtype=np.uint64))
                out["rows"][p] = [list(r) for r in _sorted(np.concatenate(parts))]
                out["n"][p] = len(rows)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["tc_grid_8", "tc_rmat_s7", "plen_rmat_s6", "sg_rmat_s7",
                                  "cspa_120", "empty_inner"])
def test_partitioned_program_on_the_cuda_engine(case, tmp_path):
    """Two gloo ranks, each running its partition on the CUDA engine (the
    engine's ternary keys, its relation table and LIE reuse across passes
    in the partitioned driver), against datalog.run on one CUDA engine:
    the same rows per head predicate, disjoint partitions, the same
    loop-pass counts."""
    world = 2
    mp.spawn(_rank_gpu, args=(world, free_port(), case, str(tmp_path)), nprocs=world, join=True)
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    text, inputs, deps = CASES[case]
    with Engine("gpu", device=0) as g:
        r = D.run(g, text, inputs(), deps=deps, sync=g.sync)
        want = {p: [list(x) for x in _sorted(rel.rows() if rel.size() else [])]
                for p, rel in r.relations.items()}
        iters = dict(r.iterations)
    for o in outs:
        assert o["iterations"] == iters
        for p in want:
            assert o["rows"][p] == want[p], p
    for p in want:
        assert sum(o["n"][p] for o in outs) == len(want[p])
