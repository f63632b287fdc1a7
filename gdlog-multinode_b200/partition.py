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

On the CUDA engine both drivers keep the exchange on the device
(`DeviceExchange`): a pass exports its candidates into a device tensor,
groups them by owner with a kernel, sends them with one all_to_all_single
of the grouped rows and loads what it receives from device memory, where
the engine sorts and deduplicates it; the host handles the per-destination
counts only.  On the oracle the rows go through the host (`route`).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch
import torch.distributed as dist

from gdlog_b200 import DELTA, FULL, INNER, NEWT, OUTER, PRED_NE, SRC, Engine


def owner(ids: np.ndarray, world: int) -> np.ndarray:
    """The rank that owns each id."""
    return (np.asarray(ids, dtype=np.int64) % world).astype(np.int64)


def _pack(rows: np.ndarray) -> torch.Tensor:
    """Rows of two ids below 2^32 as one 64-bit key each (c0 << 32 | c1),
    carried in an int64 tensor bit for bit."""
    r = np.asarray(rows, dtype=np.uint64).reshape(-1, 2)
    return torch.from_numpy(((r[:, 0] << np.uint64(32)) | r[:, 1]).view(np.int64))


def _unpack(keys: torch.Tensor) -> np.ndarray:
    k = keys.cpu().numpy().view(np.uint64)
    return np.stack([k >> np.uint64(32), k & np.uint64(0xFFFFFFFF)], axis=1)


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


class DeviceExchange:
    """A rank's exchange kept in device memory (GPU engine):
      * rows(rel, version): the version's sorted rows as an (n, 2) int64
        tensor (gdl_relation_export_device);
      * route(rows, col): every row to the owner of its column `col`
        (rows grouped by gdl_partition_rows, one all_to_all_single of the
        counts, one of the grouped rows: NCCL moves device memory directly;
        the gloo backend stages the grouped rows through host memory for
        the collective itself);
      * load(rel, rows): load_relation from device memory (sorted and
        deduplicated by the engine);
      * load_set(rel, rows): the same for rows that may repeat, loaded so
        that the relation's raw order holds each tuple once (an update
        relation's DELTA at LIE start is the first |FULL| of its rows in
        load order, src/lie.cu:49-59: a repeat would hide a tuple): the
        rows are deduplicated through a scratch relation first.
    The engine's calls return after its stream has finished; collectives
    run on torch's stream, which is synchronised before the engine reads
    their output."""

    def __init__(self, eng: Engine, world: int, device):
        self.eng, self.world = eng, world
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.nccl = dist.get_backend() == "nccl"
        self.scratch = eng.relation("_exchange_set", index_flag=False)

    def rows(self, rel, version=FULL) -> torch.Tensor:
        n = self.eng.size(rel, version)
        if n == 0:
            return torch.zeros((0, 2), dtype=torch.int64, device=self.device)
        t = torch.empty((n, 2), dtype=torch.int64, device=self.device)
        got = self.eng.export_device(rel, version, t.data_ptr(), n)
        return t[:got]

    def route(self, rows: torch.Tensor, col: int) -> torch.Tensor:
        n = rows.shape[0]
        grouped = torch.empty_like(rows)
        counts = self.eng.partition_rows(rows.data_ptr() if n else 0, n, col, self.world,
                                         grouped.data_ptr() if n else 0)
        cdev = self.device if self.nccl else "cpu"
        sc = torch.tensor(counts, dtype=torch.int64, device=cdev)
        rc = torch.empty_like(sc)
        dist.all_to_all_single(rc, sc)
        recv = rc.tolist()
        src = grouped if self.nccl else grouped.cpu()
        out = torch.empty((sum(recv), 2), dtype=torch.int64, device=src.device)
        dist.all_to_all_single(out, src, recv, counts)
        if not self.nccl:
            out = out.to(self.device)
        torch.cuda.synchronize(self.device)
        return out

    def load(self, rel, rows: torch.Tensor) -> None:
        if rows.shape[0] == 0:
            self.eng.load(rel, None)
        else:
            rows = rows.contiguous()
            self.eng.load_device(rel, rows.data_ptr(), rows.shape[0])

    def load_set(self, rel, rows: torch.Tensor) -> None:
        self.load(self.scratch, rows)
        self.load(rel, self.rows(self.scratch))


@dataclass
class PartResult:
    passes: int = 0
    full: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), dtype=np.uint64))
    per_pass_new: list = field(default_factory=list)  # global new tuples per pass


def partitioned_tc(eng: Engine, edges: np.ndarray, rank: int, world: int,
                   device=None, resident: bool | None = None) -> PartResult:
    """Transitive closure of `edges` (every rank passes the same edges) with
    path partitioned over the ranks; returns this rank's FULL partition and
    the pass count (equal on every rank).  resident (default: on the CUDA
    engine): the exchange stays on the device (DeviceExchange)."""
    if resident is None:
        resident = eng.kind == "gpu"
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
    if resident:
        x = DeviceExchange(eng, world, device)
        while True:
            res.passes += 1
            eng.load(C, None)
            join.fixpoint()
            # candidates to the owners of their first column, deduplicated
            # on the device; the new ones are the next pass's outer
            x.load_set(R, x.route(x.rows(C), 0))
            merge.fixpoint()
            new = x.rows(P, DELTA)
            x.load(D, new)
            n = torch.tensor([new.shape[0]], dtype=torch.int64,
                             device=x.device if x.nccl else "cpu")
            dist.all_reduce(n)
            res.per_pass_new.append(int(n.item()))
            if n.item() == 0:
                break
        res.full = P.rows() if P.size() else empty
        return res
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
                   device=None, resident: bool | None = None) -> PartSG:
    """Same generation of `edges` (every rank passes the same edges) with sg
    partitioned over the ranks; returns this rank's sg partition and the
    loop-pass counts of the two LIEs (equal on every rank).  resident
    (default: on the CUDA engine): the exchange stays on the device."""
    if resident is None:
        resident = eng.kind == "gpu"
    e = np.asarray(edges, dtype=np.uint64).reshape(-1, 2)
    E = eng.relation("edge_2__1_2")
    mine = e[owner(e[:, 0], world) == rank]
    eng.load(E, mine if len(mine) else None)
    sg = _Owned(eng, "sg", None)
    D = eng.relation("sg_delta")
    T = eng.relation("tmp")
    res = PartSG()
    if resident:
        return _partitioned_sg_resident(eng, E, sg, D, T, world, device, res)
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


def _partitioned_sg_resident(eng, E, sg, D, T, world, device, res) -> PartSG:
    """partitioned_sg with every pass's rows kept on the device."""
    x = DeviceExchange(eng, world, device)

    def merge(rows: torch.Tensor) -> torch.Tensor:
        # sg's update: the received rows copied into its FULL partition
        # (deduplicated first, see DeviceExchange.load_set); the new ones
        x.load_set(sg.recv, rows)
        sg.lie.fixpoint()
        return x.rows(sg.full, DELTA)

    def any_rank(n: int) -> int:
        t = torch.tensor([n], dtype=torch.int64, device=x.device if x.nccl else "cpu")
        dist.all_reduce(t)
        return int(t.item())

    init = _Join(eng, E, E, (INNER(1), OUTER(1)), pred=(PRED_NE, 0, 1), name="cand_init")
    while True:
        res.init_passes += 1
        eng.load(init.out, None)
        init.lie.fixpoint()
        new = merge(x.route(x.rows(init.out), 0))
        if any_rank(new.shape[0]) == 0:
            break
    delta = x.rows(sg.full)
    tmp_join = _Join(eng, E, D, (OUTER(1), INNER(1)), name="cand_tmp")
    sg_join = _Join(eng, E, T, (OUTER(1), INNER(1)), name="cand_sg")
    while True:
        res.passes += 1
        x.load(D, delta)
        eng.load(tmp_join.out, None)
        tmp_join.lie.fixpoint()
        x.load(T, x.route(x.rows(tmp_join.out), 0))
        eng.load(sg_join.out, None)
        sg_join.lie.fixpoint()
        delta = merge(x.route(x.rows(sg_join.out), 0))
        if any_rank(delta.shape[0]) == 0:
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


# ---------------------------------------------------------------------------
# Any program of the Datalog front end, partitioned.


def _select(rows: np.ndarray, sel: tuple) -> np.ndarray:
    """A Copy's tuple generator on the host: column SRC(c) of the source,
    plus the constant a GDL_PLUS term carries (bits 8 and up)."""
    if not len(rows):
        return np.zeros((0, len(sel)), np.uint64)
    return np.stack([rows[:, g & 0xFF] + np.uint64(g >> 8) for g in sel], axis=1)


def _route_owned(rows: np.ndarray, world: int, device) -> np.ndarray:
    """Rows of two or three columns to the owner of their first column.  A
    ternary row travels as two packed keys, (c0, c1) and (c0, c2), with the
    same destinations, so the received halves line up."""
    dest = owner(rows[:, 0], world) if len(rows) else np.zeros(0, np.int64)
    if rows.shape[1] == 2:
        return route(rows, dest, world, device)
    a = route(rows[:, :2], dest, world, device)
    b = route(rows[:, [0, 2]], dest, world, device)
    return np.concatenate([a, b[:, 1:]], axis=1)


def _keys_of(rows: np.ndarray) -> np.ndarray:
    """Packed keys of rows of two columns (one a row: c0 << 32 | c1) or
    three (two a row: (c0, c1) then (c0, c2))."""
    r = np.asarray(rows, dtype=np.uint64)
    k = (r[:, 0] << np.uint64(32)) | r[:, 1]
    if r.shape[1] == 2:
        return k
    return np.stack([k, (r[:, 0] << np.uint64(32)) | r[:, 2]], axis=1).reshape(-1)


def _rows_of(keys: np.ndarray, arity: int) -> np.ndarray:
    hi, lo = keys >> np.uint64(32), keys & np.uint64(0xFFFFFFFF)
    if arity == 2:
        return np.stack([hi, lo], axis=1)
    return np.stack([hi[0::2], lo[0::2], lo[1::2]], axis=1)


def _route_all(parts: list, world: int, device) -> list:
    """Rows of several relations (each of two or three columns) to the
    owners of their first column in one exchange: an all_to_all of a count
    for every (destination, relation) pair, then one of all the keys."""
    R = len(parts)
    counts = np.zeros((world, R), np.int64)   # keys for (destination, relation)
    chunks = [[None] * R for _ in range(world)]
    for j, rows in enumerate(parts):
        per = 1 if rows.shape[1] == 2 else 2
        dest = owner(rows[:, 0], world) if len(rows) else np.zeros(0, np.int64)
        order = np.argsort(dest, kind="stable")
        keys = _keys_of(rows[order]) if len(rows) else np.zeros(0, np.uint64)
        bounds = np.searchsorted(dest[order], np.arange(world + 1))
        for d in range(world):
            chunks[d][j] = keys[bounds[d] * per:bounds[d + 1] * per]
            counts[d, j] = len(chunks[d][j])
    send = np.concatenate([c for row in chunks for c in row]) if R else np.zeros(0, np.uint64)
    dev = device if device is not None else "cpu"
    sc = torch.from_numpy(counts.reshape(-1)).to(dev)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc)
    recv_counts = rc.cpu().numpy().reshape(world, R)
    out = torch.empty(int(recv_counts.sum()), dtype=torch.int64, device=dev)
    dist.all_to_all_single(out, torch.from_numpy(send.view(np.int64)).to(dev),
                           recv_counts.sum(axis=1).tolist(), counts.sum(axis=1).tolist())
    got = out.cpu().numpy().view(np.uint64)
    # laid out by source rank, then by relation within each source
    ends = np.cumsum(recv_counts.reshape(-1))
    starts = ends - recv_counts.reshape(-1)
    res = []
    for j, rows in enumerate(parts):
        keys = np.concatenate([got[starts[s * R + j]:ends[s * R + j]] for s in range(world)])
        res.append(_rows_of(keys, rows.shape[1]))
    return res


def _sum_all(counts: list, device) -> list:
    """Element-wise sum of a count vector over the ranks (one all_reduce)."""
    t = torch.tensor(counts, dtype=torch.int64, device=device if device is not None else "cpu")
    dist.all_reduce(t)
    return [int(x) for x in t.tolist()]


def _cat(parts: list, arity: int) -> np.ndarray:
    return np.concatenate(parts) if parts else np.zeros((0, arity), np.uint64)


class _Partition:
    """This rank's FULL partition of an updated relation, grown by the
    update step: received NEWT rows are copied into it by a one-pass LIE
    whose set difference (over arity - dependent columns,
    src/lie.cu:131-138) keeps the new ones as its DELTA."""

    def __init__(self, eng: Engine, name: str, arity: int, dep: int, rows: np.ndarray):
        self.eng, self.arity = eng, arity
        self.full = eng.relation(name, arity=arity, dependent_column_size=dep, index_flag=False)
        eng.load(self.full, rows if len(rows) else None)
        self.recv = eng.relation(name + "_recv", arity=arity, dependent_column_size=dep,
                                 index_flag=False)
        self.lie = eng.lie()
        self.lie.set_reload_full(False)
        self.lie.add_relations(self.recv, False)
        self.lie.add_relations(self.full, False)
        self.lie.add_copy(self.recv, DELTA, self.full, tuple(SRC(c) for c in range(arity)))
        self.lie.max_iteration = 0

    def rows(self) -> np.ndarray:
        return self.full.rows() if self.full.size() else np.zeros((0, self.arity), np.uint64)

    def merge(self, rows: np.ndarray) -> np.ndarray:
        # received rows deduplicated first: DELTA at LIE start is the first
        # |FULL| rows in load order (src/lie.cu:49-59), a repeat would hide one
        if len(rows):
            rows = np.unique(rows, axis=0)
        self.eng.load(self.recv, rows if len(rows) else None)
        self.lie.fixpoint()
        return self.full.rows(DELTA) if self.full.size(DELTA) else \
            np.zeros((0, self.arity), np.uint64)


@dataclass
class PartProgram:
    iterations: dict = field(default_factory=dict)  # component -> loop passes
    full: dict = field(default_factory=dict)        # head predicate -> this rank's rows
    relations: int = 0                              # engine relations used
    lies: int = 0                                   # engine LIEs used


def partitioned_program(eng: Engine, text: str, inputs: dict, rank: int, world: int,
                        deps: dict | None = None, device=None) -> PartProgram:
    """Run a Datalog program of the front end (datalog.py) with every
    relation hash-partitioned on its first column; every rank passes the
    same inputs (predicate -> rows; no row repeated, and none that a rule
    with numbers in its head also yields) and gets its
    partition of each head predicate, and the loop-pass count of each
    component, which equal those of datalog.run on one engine.

    The first column is each stored relation's join key (a swapped copy is
    stored for a join on the second), so every join reads owned keys only.
    Each component's LIE runs its ops in order, one pass at a time, as
    LIE::fixpoint_loop does (src/lie.cu:62-87):
      * a join is a one-pass LIE of the engine over the local rows of the
        versions it reads (its inner's FULL; its outer's FULL, DELTA or a
        tmp relation's NEWT); a Copy or an ACopy applies its column
        selection on the host; a Copy from FULL runs once per LIE
        (src/lie.cu:69-75);
      * rows generated into a tmp relation go at once to the owners of
        their first column (a later join of the pass reads them as its
        outer); rows generated into an updated relation stay on the rank
        that made them until the update step, which sends every updated
        relation's NEWT to the owners of their first column in one exchange
        (_route_all) and merges each into its partition on the engine (set difference and flush,
        src/lie.cu:93-198), DELTA being what was new; the loop ends when no
        rank found a tuple.
    The reference's rules on empty operands decide on global sizes (those
    of FULL and DELTA tracked from the update step's all_reduce, a NEWT's
    reduced when an op reads it): a join whose outer is empty does nothing, one whose inner
    is empty zeroes its outer's version (src/join.cu:38-45), a Copy or
    ACopy from an empty source clears its destination's NEWT
    (src/copy.cu:24-27, src/acopy.cu:14-18).  A FULL zeroed that way stays
    empty until a flush refills it, or the LIE ends (src/lie.cu:219-254)."""
    import datalog as DL
    prog = DL.compile(text, inputs.keys(), deps)
    seeds = DL.seed_rows(prog, inputs)

    def arity_of(key):
        return 3 if key[1] == 123 else 2

    def none(key):
        return np.zeros((0, arity_of(key)), np.uint64)

    def owned(rows):
        return rows[owner(rows[:, 0], world) == rank] if len(rows) else rows

    def input_rows(pred):
        return np.asarray(inputs[pred], dtype=np.uint64).reshape(-1, prog.arity[pred])

    if 3 in prog.arity.values():
        # The CUDA engine fixes the field widths of ternary keys at its first
        # ternary load, from the largest value loaded until then; one row
        # holding the largest input id, loaded first, makes them the same
        # on every rank whatever its partition holds.
        top = max((int(np.asarray(v, dtype=np.uint64).reshape(len(v), -1)[:, :2].max())
                   for v in inputs.values() if len(v)), default=0)
        ids = eng.relation("part_ids", index_flag=False)
        eng.load(ids, np.array([[top, top]], dtype=np.uint64))

    parts = {}       # updated (predicate, order) -> _Partition
    static = {}      # (predicate, order) read from outside a component -> engine relation
    host_full = {}   # (predicate, order) -> this rank's FULL rows
    zero_full = set()
    full_gen = {}    # updated key -> how many times its FULL changed
    gfull = {}       # (predicate, order) -> its FULL's size over all ranks
    scratch = {}     # operand slot -> [relation, what it holds]
    outs = {}
    lies = {}
    res = PartProgram()

    def full_rows(key):
        return none(key) if key in zero_full else host_full[key]

    def operand(slot, key, token, rows):
        """An engine relation holding `rows` (one per operand slot, loaded
        again only when what it should hold changed)."""
        if slot not in scratch:
            name = f"{DL._rel_name(*key) if not key[0].startswith('tmp_') else key[0]}_{slot[1]}"
            scratch[slot] = [DL.new_relation(eng, prog, key, name=name), None]
        rel, held = scratch[slot]
        if held != token:
            eng.load(rel, rows if len(rows) else None)
            scratch[slot][1] = token
        return rel

    def inner_of(key):
        if key in static:
            return static[key]
        return operand((key, "full"), key, ("full", full_gen[key]), host_full[key])

    for C in prog.comps:
        for key in C.statics:
            if key in static:
                continue
            pred, order = key
            if pred in inputs:
                rows = input_rows(pred)
                rows = owned(rows[:, ::-1].copy() if order == 21 else rows)
            else:  # a lower component's predicate: swapped rows go to new owners
                base = full_rows((pred, prog.main[pred]))
                rows = _route_owned(base[:, ::-1].copy(), world, device) if order == 21 else base
                if order == 21 and len(rows):
                    rows = np.unique(rows, axis=0)
            rel = DL.new_relation(eng, prog, key)
            eng.load(rel, rows if len(rows) else None)
            static[key] = rel
            host_full[key] = rel.rows() if rel.size() else none(key)

        def start(key, rows):
            name = DL._rel_name(*key) + "_part"
            parts[key] = _Partition(eng, name, arity_of(key), prog.deps.get(key[0], 0)
                                    if key[1] == 123 else 0, rows)
            host_full[key] = parts[key].rows()
            full_gen[key] = 0

        for p in C.preds:
            key = (p, prog.main[p])
            rows = [input_rows(p)] if p in inputs else []
            rows = owned(_cat(rows + seeds.get(p, []), prog.arity[p]))
            start(key, rows)
        for key in C.update:
            if key in parts:
                continue
            # a swapped mirror: the predicate's loaded rows, to their new owners
            base = host_full[(key[0], prog.main[key[0]])]
            start(key, _route_owned(base[:, ::-1].copy(), world, device))
        if not C.ops:
            continue
        # global sizes of the FULLs the component reads, one all_reduce; the
        # update step's all_reduce keeps them (and DELTA's) current, so
        # only NEWT sizes need one when an op reads them
        fresh = [k for k in C.statics if k not in gfull] + list(C.update)
        for k, n in zip(fresh, _sum_all([len(host_full[k]) for k in fresh], device)):
            gfull[k] = n
        # LIE start: DELTA := FULL (src/lie.cu:49-59; inputs without repeats)
        delta = {key: host_full[key] for key in C.update}
        gdelta = {key: gfull[key] for key in C.update}
        copied = set()
        it = 0
        while True:
            it += 1
            newt = {key: [] for key in C.update + C.tmps}
            zero_delta = set()

            def placed(key, rows):
                # a tmp relation's NEWT is read as a join's outer in this
                # pass, so it goes to the owners of its join key now; an
                # updated relation's NEWT is read only by ACopies (which
                # route what they write) and by the update step, so its rows
                # stay where they were generated and travel once, there
                return _route_owned(rows, world, device) if key in C.tmps else rows

            def global_sizes(*reads):
                """Sizes over all ranks of (key, version, local rows) reads:
                FULL and DELTA from the tracked sizes, NEWT by all_reduce."""
                out = [None if ver == NEWT else
                       0 if (key in zero_delta if ver == DELTA else key in zero_full) else
                       (gdelta if ver == DELTA else gfull)[key] for key, ver, _ in reads]
                ask = [i for i, x in enumerate(out) if x is None]
                if ask:
                    for i, n in zip(ask, _sum_all([len(reads[i][2]) for i in ask], device)):
                        out[i] = n
                return out

            def version(key, ver):
                if ver == DELTA:
                    return none(key) if key in zero_delta else delta[key]
                if ver == NEWT:
                    return _cat(newt[key], arity_of(key))
                return full_rows(key)

            for i, op in enumerate(C.ops):
                if op.kind == "copy" and op.src_ver == FULL:
                    if i in copied:
                        continue
                    copied.add(i)
                if op.kind == "acopy":
                    # NEWT replaced by the selection of the source's NEWT
                    # (cleared when that is empty everywhere, which is the
                    # same): no size to agree on
                    newt[op.out] = [placed(op.out, _select(version(op.src, NEWT), op.sel))]
                    continue
                if op.kind == "copy":
                    src = version(op.src, op.src_ver)
                    if global_sizes((op.src, op.src_ver, src))[0] == 0:
                        newt[op.out] = []
                        continue
                    newt[op.out].append(placed(op.out, _select(src, op.sel)))
                    continue
                if op.src_ver != FULL:
                    raise ValueError("a join's inner is read as FULL")
                rin = version(op.src, op.src_ver)
                rout = version(op.outer, op.outer_ver)
                n_in, n_out = global_sizes((op.src, op.src_ver, rin),
                                           (op.outer, op.outer_ver, rout))
                if n_out == 0:
                    continue
                if n_in == 0:
                    if op.outer_ver == DELTA:
                        zero_delta.add(op.outer)
                    elif op.outer_ver == NEWT:
                        newt[op.outer] = []
                    else:
                        zero_full.add(op.outer)
                    continue
                got = none(op.out)
                if len(rin) and len(rout):
                    inner = inner_of(op.src)
                    if op.outer_ver == FULL:
                        outer = inner_of(op.outer)
                    else:
                        tok = (it, i) if op.outer_ver == NEWT else ("delta", it)
                        outer = operand((op.outer, "delta" if op.outer_ver == DELTA else "newt"),
                                        op.outer, tok, rout)
                    a = arity_of(op.out)
                    if a not in outs:
                        outs[a] = eng.relation(f"part_out{a}", arity=a, index_flag=False)
                    lkey = (i, C.name)
                    if lkey not in lies:
                        lie = eng.lie()
                        lie.add_relations(inner, True)
                        if outer is not inner:
                            lie.add_relations(outer, True)
                        lie.add_relations(outs[a], False)
                        kw = {"pred": op.pred} if op.pred else {}
                        lie.add_join(inner, FULL, outer, FULL, outs[a], op.sel, **kw)
                        lie.max_iteration = 0
                        lies[lkey] = (lie, inner, outer)
                    lie, bi, bo = lies[lkey]
                    assert bi is inner and bo is outer
                    eng.load(outs[a], None)
                    lie.fixpoint()
                    got = outs[a].rows() if outs[a].size() else got
                newt[op.out].append(placed(op.out, got))
            # the update step (src/lie.cu:93-198)
            new = []
            sent = _route_all([_cat(newt[key], arity_of(key)) for key in C.update], world,
                              device)
            for key, rows in zip(C.update, sent):
                delta[key] = parts[key].merge(rows) if len(rows) else none(key)
                new.append(len(delta[key]))
            grew = _sum_all(new, device)
            for key, n, n_all in zip(C.update, new, grew):
                if n:  # DELTA is disjoint from FULL: the flushed FULL is their union
                    host_full[key] = np.concatenate([host_full[key], delta[key]])
                    full_gen[key] += 1
                gfull[key] += n_all
                gdelta[key] = n_all
                if n_all:
                    zero_full.discard(key)
            if sum(grew) == 0:
                break
        for key in C.update:  # LIE end: FULL flattened again (src/lie.cu:219-254)
            zero_full.discard(key)
        res.iterations[C.name] = it
    for C in prog.comps:
        for p in C.preds:
            res.full[p] = host_full[(p, prog.main[p])]
    res.relations = len(eng.relations)
    res.lies = len(lies) + len(parts)
    return res


def run_file_partitioned(eng: Engine, path: str, rank: int, world: int,
                         facts_dir: str | None = None, out_dir: str | None = None,
                         inputs: dict | None = None, device=None) -> tuple:
    """datalog.run_file with every relation partitioned over the ranks:
    each rank reads the inputs (repeated rows dropped, as the reference's
    load does, src/relation.cu:570-593) and runs its partition; rank 0
    writes each `.output` relation (the union of the partitions, sorted,
    tab-separated) to <out_dir>/<name>.csv.  Returns (PartProgram,
    {name: size} for the `.printsize` relations), the sizes on every rank."""
    import os

    import datalog as DL
    from gdlog_b200 import write_tsv
    text, d, given = DL.read_program(path, facts_dir, inputs)
    given = {k: np.unique(np.asarray(v, dtype=np.uint64).reshape(len(v), -1), axis=0)
             for k, v in given.items()}
    res = partitioned_program(eng, text, given, rank, world, deps=d.dep, device=device)
    names = sorted(d.printsize)
    counts = _sum_all([len(res.full[n]) if n in res.full else 0 for n in names], device)
    sizes = {n: c if n in res.full else DL.input_size(given, n) for n, c in zip(names, counts)}
    if out_dir:
        if rank == 0:
            os.makedirs(out_dir, exist_ok=True)
        for n in d.outputs:
            parts = [None] * world
            dist.all_gather_object(parts, res.full.get(n))
            if rank:
                continue
            rows = np.concatenate(parts) if n in res.full else given[n]
            rows = rows[np.lexsort(rows.T[::-1])] if len(rows) else rows
            write_tsv(os.path.join(out_dir, n + ".csv"), rows)
    return res, sizes
