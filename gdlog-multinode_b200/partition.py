"""Partitioned fixpoint: one relation split across ranks (one GPU each).

The reference runs a LIE's semi-naive loop (src/lie.cu:26-274) on one GPU.
Here transitive closure, path(x, z) :- edge(x, y), path(y, z) as the
reference's driver writes it (test/tc.cu:80-149), runs over `world` ranks
with every relation hash-partitioned on its join column.  Rank r owns the
ids v with v % world == r:
  * edge tuples (x, y) whose y it owns, kept as edge_2__2_1 rows (y, x) —
    the join's inner, indexed on the join column;
  * path tuples (a, b) whose a it owns: its FULL partition, and DELTA, the
    tuples it found new in the last pass.
One pass on rank r:
  1. the local join of the edge partition with DELTA (both sides hold only
     owned join values, so nothing is missed) gives candidates (x, z): one
     fixpoint pass of the engine over the local partition;
  2. each candidate goes to owner(x): one all_to_all_single of packed keys
     (x << 32 | z; the NCCL backend over NVLink, gloo on the host);
  3. the owner keeps the candidates not yet in its FULL partition (an
     engine Copy into FULL: the update step deduplicates and yields DELTA);
     both steps are one-pass LIEs built once and run every pass;
  4. an all_reduce of the new-tuple counts ends the loop when no rank found
     any, so every rank takes the same collective steps.
Each pass extends the paths by one edge, as the single-GPU loop does, so the
pass count equals its loop-pass count and the union of the FULL partitions
is its closure.  The engine on each rank is any gdlog_b200.Engine.

Same generation (test/sg.cu:93-191) partitions the same way: edge and sg
on their first column (sg(a, b) with a owned), so both joins of a pass —
tmp(b, x) :- edge(a, x), sg(a, b) and sg(x, y) :- edge(b, y), tmp(b, x) —
read only owned keys; a pass routes tmp candidates to owner(b), then sg
candidates to owner(x).  Its non-recursive rule sg(x, y) :- edge(p, x),
edge(p, y), x != y runs as its own loop, as the driver's first LIE does.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch
import torch.distributed as dist

from gdlog_b200 import DELTA, FULL, INNER, OUTER, PRED_NE, SRC, Engine


def owner(ids: np.ndarray, world: int) -> np.ndarray:
    """The rank that owns each id."""
    return (np.asarray(ids, dtype=np.int64) % world).astype(np.int64)


def _pack(rows: np.ndarray) -> torch.Tensor:
    r = np.asarray(rows, dtype=np.int64).reshape(-1, 2)
    return torch.from_numpy((r[:, 0] << 32) | r[:, 1])


def _unpack(keys: torch.Tensor) -> np.ndarray:
    k = keys.cpu().numpy().astype(np.int64)
    return np.stack([k >> 32, k & 0xFFFFFFFF], axis=1).astype(np.uint64)


def route(rows: np.ndarray, dest: np.ndarray, world: int, device=None) -> np.ndarray:
    """Send row i to rank dest[i]; return the rows this rank receives (one
    all_to_all of the counts, one of the packed keys)."""
    order = np.argsort(dest, kind="stable")
    keys = _pack(rows[order]) if len(rows) else torch.zeros(0, dtype=torch.int64)
    send_counts = torch.from_numpy(np.bincount(dest, minlength=world).astype(np.int64))
    recv_counts = torch.empty(world, dtype=torch.int64)
    if device is not None:
        keys, send_counts, recv_counts = keys.to(device), send_counts.to(device), recv_counts.to(device)
    dist.all_to_all_single(recv_counts, send_counts)
    out = torch.empty(int(recv_counts.sum().item()), dtype=torch.int64, device=keys.device)
    dist.all_to_all_single(out, keys, recv_counts.tolist(), send_counts.tolist())
    return _unpack(out)


@dataclass
class PartResult:
    passes: int = 0
    full: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), dtype=np.uint64))
    per_pass_new: list = field(default_factory=list)  # global new tuples per pass


def partitioned_tc(eng: Engine, edges: np.ndarray, rank: int, world: int,
                   device=None) -> PartResult:
    """Transitive closure of `edges` (every rank passes the same edges) with
    path partitioned over the ranks; returns this rank's FULL partition and
    the pass count (equal on every rank)."""
    e = np.asarray(edges, dtype=np.uint64).reshape(-1, 2)
    mine_e = e[owner(e[:, 1], world) == rank]
    mine_p = e[owner(e[:, 0], world) == rank]
    E = eng.relation("edge_2__2_1")
    eng.load(E, mine_e[:, ::-1].copy() if len(mine_e) else None)
    P = eng.relation("path_full", index_flag=False)
    eng.load(P, mine_p if len(mine_p) else None)
    D = eng.relation("path_delta")
    eng.load(D, mine_p if len(mine_p) else None)
    C = eng.relation("path_cand", index_flag=False)
    R = eng.relation("path_recv", index_flag=False)
    # one pass each (max_iteration 0), the same two LIEs every pass
    join = eng.lie()
    join.add_relations(E, True)
    join.add_relations(D, True)
    join.add_relations(C, False)
    join.add_join(E, FULL, D, FULL, C, (INNER(1), OUTER(1)))
    join.max_iteration = 0
    # a Copy from R's DELTA (R's rows at every LIE start, src/lie.cu:49-59;
    # a Copy from FULL would run once per LIE, src/copy.cu) into P: P's
    # update step deduplicates, and its DELTA is what was new
    merge = eng.lie()
    merge.set_reload_full(False)
    merge.add_relations(R, False)
    merge.add_relations(P, False)
    merge.add_copy(R, DELTA, P, (SRC(0), SRC(1)))
    merge.max_iteration = 0
    res = PartResult()
    empty = np.zeros((0, 2), dtype=np.uint64)
    while True:
        res.passes += 1
        # 1. candidates of the local join
        eng.load(C, None)
        join.fixpoint()
        cand = C.rows() if C.size() else empty
        # 2. to the owners of their first column
        got = route(cand, owner(cand[:, 0], world) if len(cand) else np.zeros(0, np.int64),
                    world, device)
        # 3. the new ones (received rows deduplicated first: an update
        # relation's DELTA at LIE start is the first |FULL| of its rows in
        # load order, src/lie.cu:49-59, so a repeat would hide a tuple)
        if len(got):
            got = np.unique(got, axis=0)
        eng.load(R, got if len(got) else None)
        merge.fixpoint()
        new = P.rows(DELTA) if P.size(DELTA) else empty
        eng.load(D, new if len(new) else None)
        # 4. stop when no rank found a new tuple
        n = torch.tensor([len(new)], dtype=torch.int64,
                         device=device if device is not None else "cpu")
        dist.all_reduce(n)
        res.per_pass_new.append(int(n.item()))
        if n.item() == 0:
            break
    res.full = P.rows() if P.size() else np.zeros((0, 2), dtype=np.uint64)
    return res


class _Owned:
    """A relation partition that grows by deduplicated merges: received rows
    are copied into it by a one-pass LIE whose update step keeps the new
    ones (its DELTA)."""

    def __init__(self, eng: Engine, name: str, rows):
        self.eng = eng
        self.full = eng.relation(name, index_flag=False)
        eng.load(self.full, rows if rows is not None and len(rows) else None)
        self.recv = eng.relation(name + "_recv", index_flag=False)
        # a Copy from the received relation's DELTA (its rows at every LIE
        # start, src/lie.cu:49-59; a Copy from FULL would run once per LIE)
        self.lie = eng.lie()
        self.lie.set_reload_full(False)
        self.lie.add_relations(self.recv, False)
        self.lie.add_relations(self.full, False)
        self.lie.add_copy(self.recv, DELTA, self.full, (SRC(0), SRC(1)))
        self.lie.max_iteration = 0

    def merge(self, rows: np.ndarray) -> np.ndarray:
        """Add rows; return those that were not there yet.  Rows are
        deduplicated first: a relation's DELTA at LIE start is the first
        |FULL| of its rows in load order, so a repeat would hide a tuple."""
        if len(rows):
            rows = np.unique(rows, axis=0)
        self.eng.load(self.recv, rows if len(rows) else None)
        self.lie.fixpoint()
        return self.full.rows(DELTA) if self.full.size(DELTA) else np.zeros((0, 2), np.uint64)

    def rows(self) -> np.ndarray:
        return self.full.rows() if self.full.size() else np.zeros((0, 2), np.uint64)


class _Join:
    """One join of the partitioned program as a one-pass LIE: the inner's
    FULL joined with the outer's FULL into a candidates relation."""

    def __init__(self, eng: Engine, inner, outer, sel, pred=None, name="cand"):
        self.eng = eng
        self.out = eng.relation(name, index_flag=False)
        self.lie = eng.lie()
        self.lie.add_relations(inner, True)
        if outer is not inner:
            self.lie.add_relations(outer, True)
        self.lie.add_relations(self.out, False)
        if pred is None:
            self.lie.add_join(inner, FULL, outer, FULL, self.out, sel)
        else:
            self.lie.add_join(inner, FULL, outer, FULL, self.out, sel, pred=pred)
        self.lie.max_iteration = 0

    def run(self) -> np.ndarray:
        self.eng.load(self.out, None)
        self.lie.fixpoint()
        return self.out.rows() if self.out.size() else np.zeros((0, 2), np.uint64)


def _to_owners(rows: np.ndarray, col: int, world: int, device) -> np.ndarray:
    dest = owner(rows[:, col], world) if len(rows) else np.zeros(0, np.int64)
    return route(rows, dest, world, device)


def _any(n: int, device) -> int:
    t = torch.tensor([n], dtype=torch.int64, device=device if device is not None else "cpu")
    dist.all_reduce(t)
    return int(t.item())


@dataclass
class PartSG:
    init_passes: int = 0
    passes: int = 0
    full: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), dtype=np.uint64))


def partitioned_sg(eng: Engine, edges: np.ndarray, rank: int, world: int,
                   device=None) -> PartSG:
    """Same generation of `edges` (every rank passes the same edges) with sg
    partitioned over the ranks; returns this rank's sg partition and the
    loop-pass counts of the two LIEs (equal on every rank)."""
    e = np.asarray(edges, dtype=np.uint64).reshape(-1, 2)
    E = eng.relation("edge_2__1_2")
    mine = e[owner(e[:, 0], world) == rank]
    eng.load(E, mine if len(mine) else None)
    sg = _Owned(eng, "sg", None)
    D = eng.relation("sg_delta")
    T = eng.relation("tmp")
    res = PartSG()
    # sg(x, y) :- edge(p, x), edge(p, y), x != y: its own loop (the second
    # pass finds nothing new, as the driver's first LIE does)
    init = _Join(eng, E, E, (INNER(1), OUTER(1)), pred=(PRED_NE, 0, 1), name="cand_init")
    while True:
        res.init_passes += 1
        new = sg.merge(_to_owners(init.run(), 0, world, device))
        if _any(len(new), device) == 0:
            break
    # the recursive rules, from DELTA = FULL (src/lie.cu:49-59)
    delta = sg.rows()
    tmp_join = _Join(eng, E, D, (OUTER(1), INNER(1)), name="cand_tmp")
    sg_join = _Join(eng, E, T, (OUTER(1), INNER(1)), name="cand_sg")
    while True:
        res.passes += 1
        eng.load(D, delta if len(delta) else None)
        # tmp(b, x) :- edge(a, x), sg(a, b): to owner(b)
        tmp = _to_owners(tmp_join.run(), 0, world, device)
        if len(tmp):
            tmp = np.unique(tmp, axis=0)
        eng.load(T, tmp if len(tmp) else None)
        # sg(x, y) :- edge(b, y), tmp(b, x): to owner(x), deduplicated there
        delta = sg.merge(_to_owners(sg_join.run(), 0, world, device))
        if _any(len(delta), device) == 0:
            break
    res.full = sg.rows()
    return res


def gather_rows(rows: np.ndarray, world: int) -> np.ndarray:
    """Every rank's rows on every rank, sorted (the union of the partitions)."""
    parts = [None] * world
    dist.all_gather_object(parts, np.asarray(rows, dtype=np.uint64))
    allr = np.concatenate([p.reshape(-1, 2) for p in parts]) if parts else np.zeros((0, 2))
    order = np.lexsort((allr[:, 1], allr[:, 0]))
    return allr[order]
