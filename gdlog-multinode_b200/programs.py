"""The three Datalog programs of the reference, as operator programs.

Each function builds the same relations, LIEs and RA operators, in the same
order, as the reference's hand-compiled driver, and runs them on an Engine
(GPU or oracle):

* ``tc``   – test/tc.cu:80-149   (path(x,z) :- edge(x,y), path(y,z); left
                                   linear, reload_full_flag = false)
* ``sg``   – test/sg.cu:93-191   (init SCC + recursive SCC with a tmp
                                   relation)
* ``cspa`` – test/cspa.cu:100-379 (init SCC of 7 copies + analysis SCC of
                                   11 joins and 2 ACopies, 3 tmp relations)
* ``path_length`` – test/path_length.cu:59-140 (path(a, y, l + 1) :-
                                   edge(a, x), path(x, y, l); arity 3 with a
                                   dependent length column)

The hooks of the drivers are pure column selections; they are written here
in the C-ABI encoding (INNER(c) / OUTER(c) / SRC(c)):
  reorder_path  newt = (inner[1], outer[1])   test/tc.cu:61-65
  reorder_path1 newt = (outer[1], inner[1])   test/sg.cu:66-70
  join_10_11    out  = (outer[1], inner[1])   test/cspa.cu:84-88
  join_01_11    out  = (inner[1], outer[1])   test/cspa.cu:91-95
  cp_1 / cp_2_1__1_2   (src[1], src[0])       test/tc.cu:74-77, cspa.cu:73-76
  cp_2_1__1            (src[0], src[0])       test/cspa.cu:62-65
  cp_2_1__2            (src[1], src[1])       test/cspa.cu:67-70
  tuple_pred_eq_11     t[0] != t[1]           test/sg.cu:88
and path_length's computing hook in the PLUS encoding:
  reorder_path  newt = (inner[1], outer[1], outer[2] + 1)   test/path_length.cu:52-57
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from gdlog_b200 import (DELTA, FULL, INNER, NEWT, OUTER, PRED_NE, SRC, Engine,
                        Relation, PLUS)
from workloads import reverse

REORDER_PATH = (INNER(1), OUTER(1))
REORDER_PATH1 = (OUTER(1), INNER(1))
JOIN_10_11 = (OUTER(1), INNER(1))
JOIN_01_11 = (INNER(1), OUTER(1))
CP_SWAP = (SRC(1), SRC(0))
CP_2_1__1 = (SRC(0), SRC(0))
CP_2_1__2 = (SRC(1), SRC(1))


@dataclass
class Result:
    """Outcome of one program run: the relation(s) the driver reports, the
    iteration count of each LIE, and the fixpoint wall seconds."""
    relations: dict = field(default_factory=dict)
    iterations: dict = field(default_factory=dict)
    seconds: float = 0.0
    lies: dict = field(default_factory=dict)

    @property
    def output(self) -> Relation:
        return next(iter(self.relations.values()))


def tc(eng: Engine, edges: np.ndarray, sync=None) -> Result:
    """test/tc.cu:80-149."""
    edge_2__2_1 = eng.relation("edge_2__2_1")
    path_2__1_2 = eng.relation("path_2__1_2", index_flag=False)
    eng.load(path_2__1_2, edges)
    eng.load(edge_2__2_1, reverse(edges))
    lie = eng.lie()
    lie.set_reload_full(False)
    lie.add_relations(edge_2__2_1, True)
    lie.add_relations(path_2__1_2, False)
    lie.add_join(edge_2__2_1, FULL, path_2__1_2, DELTA, path_2__1_2, REORDER_PATH)
    t0 = time.perf_counter()
    it = lie.fixpoint()
    if sync:
        sync()
    r = Result(seconds=time.perf_counter() - t0)
    r.relations["path"] = path_2__1_2
    r.iterations["tc"] = it
    r.lies["tc"] = lie
    return r


def sg(eng: Engine, edges: np.ndarray, sync=None) -> Result:
    """test/sg.cu:93-191."""
    edge_2__1_2 = eng.relation("edge_2__1_2")
    edge_2__2_1 = eng.relation("edge_2__2_1")
    eng.load(edge_2__2_1, reverse(edges))
    sg_2__1_2 = eng.relation("sg_2__2_1", index_flag=False)
    eng.load(sg_2__1_2, None)
    eng.load(edge_2__1_2, edges)
    t0 = time.perf_counter()
    init = eng.lie()
    init.add_relations(edge_2__1_2, True)
    init.add_relations(sg_2__1_2, False)
    # sg(x, y) :- edge(p, x), edge(p, y), x != y.
    init.add_join(edge_2__1_2, FULL, edge_2__1_2, FULL, sg_2__1_2, REORDER_PATH,
                  pred=(PRED_NE, 0, 1))
    it0 = init.fixpoint()
    tmp = eng.relation("tmp", index_flag=False)
    eng.load(tmp, None)
    lie = eng.lie()
    lie.add_relations(edge_2__1_2, True)
    lie.add_relations(sg_2__1_2, False)
    lie.add_tmp_relation(tmp)
    # tmp(b, x) :- edge(a, x), sg(a, b).
    lie.add_join(edge_2__1_2, FULL, sg_2__1_2, DELTA, tmp, REORDER_PATH1)
    # sg(x, y) :- edge(b, y), tmp(b, x).
    lie.add_join(edge_2__1_2, FULL, tmp, NEWT, sg_2__1_2, REORDER_PATH1)
    it1 = lie.fixpoint()
    if sync:
        sync()
    r = Result(seconds=time.perf_counter() - t0)
    r.relations["sg"] = sg_2__1_2
    r.iterations.update(init=it0, sg=it1)
    r.lies.update(init=init, sg=lie)
    return r


def cspa(eng: Engine, assign: np.ndarray, deref: np.ndarray, sync=None) -> Result:
    """test/cspa.cu:100-379."""
    assign_2__2_1 = eng.relation("assign_2__2_1")
    eng.load(assign_2__2_1, reverse(assign))
    dereference_2__1_2 = eng.relation("dereference_2__1_2")
    eng.load(dereference_2__1_2, deref)
    dereference_2__2_1 = eng.relation("dereference_2__2_1")
    eng.load(dereference_2__2_1, reverse(deref))
    vf12 = eng.relation("value_flow_2__1_2")
    eng.load(vf12, None)
    vf21 = eng.relation("value_flow_2__2_1")
    eng.load(vf21, None)
    ma12 = eng.relation("memory_alias_2__1_2")
    eng.load(ma12, None)
    ma21 = eng.relation("memory_alias_2__2_1")
    eng.load(ma21, None)

    t0 = time.perf_counter()
    init = eng.lie()
    for rel in (vf12, vf21, ma12, ma21):
        init.add_relations(rel, False)
    init.add_relations(assign_2__2_1, True)
    init.add_copy(assign_2__2_1, FULL, vf12, CP_2_1__1)
    init.add_copy(assign_2__2_1, FULL, vf12, CP_2_1__2)
    init.add_copy(assign_2__2_1, FULL, vf12, CP_SWAP)
    init.add_copy(assign_2__2_1, FULL, ma12, CP_2_1__1)
    init.add_copy(assign_2__2_1, FULL, ma12, CP_2_1__2)
    init.add_copy(vf12, DELTA, vf21, CP_SWAP)
    init.add_copy(ma12, DELTA, ma21, CP_SWAP)
    it0 = init.fixpoint()

    vff12 = eng.relation("value_flow_forward_2__1_2")
    eng.load(vff12, None)
    vff21 = eng.relation("value_flow_forward_2__2_1")
    eng.load(vff21, None)
    va12 = eng.relation("value_alias_2__1_2", index_flag=False)
    eng.load(va12, None)
    tmp_def = eng.relation("tmp_rel_def", index_flag=False)
    eng.load(tmp_def, None)
    tmp_ma1 = eng.relation("tmp_rel_ma1", index_flag=False, tmp_flag=True)
    eng.load(tmp_ma1, None)
    tmp_ma2 = eng.relation("tmp_rel_ma2", index_flag=False, tmp_flag=True)
    eng.load(tmp_ma2, None)

    lie = eng.lie()
    lie.add_relations(assign_2__2_1, True)
    lie.add_relations(dereference_2__1_2, True)
    lie.add_relations(dereference_2__2_1, True)
    for rel in (vf12, vf21, ma12, ma21, va12):
        lie.add_relations(rel, False)
    for rel in (tmp_def, tmp_ma1, tmp_ma2):
        lie.add_tmp_relation(rel)
    # ValueFlow(x, y) :- ValueFlow(x, z), ValueFlow(z, y).
    lie.add_join(vf12, FULL, vf21, DELTA, vf12, JOIN_10_11)
    lie.add_join(vf21, FULL, vf12, DELTA, vf12, JOIN_01_11)
    # ValueAlias(x, y) :- ValueFlow(z, x), ValueFlow(z, y).
    lie.add_join(vf12, FULL, vf12, DELTA, va12, JOIN_01_11)
    lie.add_join(vf12, FULL, vf12, DELTA, va12, JOIN_10_11)
    # ValueFlow(x, y) :- Assign(x, z), MemoryAlias(z, y).
    lie.add_join(assign_2__2_1, FULL, ma12, DELTA, vf12, JOIN_01_11)
    # tmp_rel_def(z, x) :- Dereference(y, x), ValueAlias(y, z).
    lie.add_join(dereference_2__1_2, FULL, va12, DELTA, tmp_def, JOIN_10_11)
    # MemoryAlias(x, w) :- Dereference(z, w), tmp_rel_def(z, x).
    lie.add_join(dereference_2__1_2, FULL, tmp_def, NEWT, ma12, JOIN_10_11)
    # ValueAlias(x, y) :- ValueFlow(z, x), MemoryAlias(z, w), ValueFlow(w, y).
    lie.add_join(ma12, FULL, vf12, DELTA, tmp_ma1, JOIN_01_11)
    lie.add_join(vf12, FULL, ma12, DELTA, tmp_ma1, JOIN_10_11)
    lie.add_join(vf12, FULL, tmp_ma1, NEWT, va12, JOIN_10_11)
    lie.add_join(ma21, FULL, vf12, DELTA, tmp_ma2, JOIN_01_11)
    lie.add_join(vf12, FULL, tmp_ma2, NEWT, va12, JOIN_01_11)
    lie.add_acopy(vf12, vf21, CP_SWAP)
    lie.add_acopy(ma12, ma21, CP_SWAP)
    it1 = lie.fixpoint()
    if sync:
        sync()
    r = Result(seconds=time.perf_counter() - t0)
    r.relations.update(value_flow=vf12, memory_alias=ma12, value_alias=va12)
    r.iterations.update(init=it0, analysis=it1)
    r.lies.update(init=init, analysis=lie)
    return r


def path_length(eng: Engine, edges: np.ndarray, sync=None) -> Result:
    """test/path_length.cu:59-140: path(x, y, 1) for every edge, then
    path(a, y, l + 1) :- edge(a, x), path(x, y, l), where a (x, y) pair is
    new only if no path(x, y, _) exists yet (dependent_column_size 1), so
    the lengths are the shortest in edges."""
    e = np.asarray(edges, dtype=np.uint64)
    rows = np.concatenate([e, np.ones((len(e), 1), dtype=np.uint64)], axis=1) if len(e) else \
        np.zeros((0, 3), dtype=np.uint64)
    edge_2__2_1 = eng.relation("edge_2__2_1")
    path_3__1_2_3 = eng.relation("path_3__1_2_3", arity=3, dependent_column_size=1,
                                 index_flag=False)
    eng.load(path_3__1_2_3, rows)
    eng.load(edge_2__2_1, reverse(e))
    t0 = time.perf_counter()
    lie = eng.lie()
    lie.add_relations(edge_2__2_1, True)
    lie.add_relations(path_3__1_2_3, False)
    lie.add_join(edge_2__2_1, FULL, path_3__1_2_3, DELTA, path_3__1_2_3,
                 (INNER(1), OUTER(1), PLUS(OUTER(2), 1)))
    it = lie.fixpoint()
    if sync:
        sync()
    r = Result(seconds=time.perf_counter() - t0)
    r.relations["path"] = path_3__1_2_3
    r.iterations["plen"] = it
    r.lies["plen"] = lie
    return r
