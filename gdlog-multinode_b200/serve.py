"""Serving loop: continuous batching of Datalog queries on one GPU.

A stream of queries (each carrying its own graph; transitive closure or
same generation, as in the reference's drivers test/tc.cu and test/sg.cu)
arrives over time.  The server keeps `slots` engines, each with its own
CUDA stream.  Whenever a slot is free it takes, from the queue in arrival
order, every waiting query of one program kind that fits the slot's HBM
budget, and runs them as ONE batched fixpoint (batch.py: block-diagonal
bitmaps, all instances in the same kernels).  Queries that arrive while
other batches are on the GPU are admitted as soon as a slot and memory
free up, and their kernels overlap with the batches in flight (other
streams).  Relations live on the device from load to result.

Admission uses an HBM estimate per query that can join a batch: the
bitmaps of its relations (n^2 / 8 bytes each, three per updated relation
plus NEWT of the tmp relation) plus 16 bytes per candidate of its first
join.  The candidates
come from that join's count pass on the device (gdl_join_count: the
query's relations are loaded into an estimator engine as its program loads
them, and k_join_count sums, per outer row, the length of the inner run it
probes), taken as each query arrives; `hbm_estimate` derives the same count
from the graph's degrees on the host and serves as its cross-check and for
streams that are not served on a GPU.  The same candidate count
bounds the largest list the batch's first fixpoint hands to the next one,
so a batch is also capped at half of the engine's list limit (2^30 rows)
in summed candidates.  Later iterations can still outgrow a list (a batch of
same-generation queries grows fast); a batch the engine refuses for size
(GDL_E_UNSUPPORTED list limit, GDL_E_NOMEM) is split in halves and each half
run again, down to single queries.

A query on 2^12 or more nodes is served alone through the plain engine
instead (`plain_min_nodes`), and so is a batch that holds one query: there
the joins run gathered by output row or along the inner's in-edges
(csrc/pull.cuh), which the block-diagonal batched layout does not have, so
one query runs faster alone than as a batch of one, and a large query no
longer sets the pace of a batch of small ones.  Batches form when queries
queue up behind the slots.

The plain baseline serves the same stream one query at a time through the
plain (unbatched) engine.  Both report p50 / p99 latency (finish - arrival)
and throughput, and every query's result (size, digest of its sorted tuples
in local ids, loop passes) so that results can be checked alone vs. mixed.
"""
from __future__ import annotations

import argparse
import collections
import json
import threading
import time
from dataclasses import dataclass, field

import numpy as np

import batch as B
import programs as P
import workloads as W
from gdlog_b200 import FULL, Engine, GdlError

# gdl_status codes of a batch too large for the engine (include/gdlog_b200.h)
_TOO_LARGE = (3, 4)  # GDL_E_NOMEM, GDL_E_UNSUPPORTED

PROGRAMS = {"tc": P.tc, "sg": P.sg}


@dataclass
class Request:
    id: int
    kind: str
    inputs: tuple
    nodes: int
    arrival: float
    est_bytes: int = 0
    est_tuples: int = 0
    start: float = -1.0
    finish: float = -1.0
    result: object = None


def make_stream(n=20000, rate=200.0, tc_frac=0.7, seed=7, max_scale=14, min_scale=10,
                l_range=(8, 128), w_range=(16, 256)):
    """Poisson arrivals; 70% TC on a layered DAG (L, W log-uniform in
    l_range x w_range), 30% SG on an R-MAT graph of scale
    U{min_scale..max_scale} with 4 x nodes edges."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    reqs = []
    for i in range(n):
        if rng.random() < tc_frac:
            L = W.log_uniform_int(rng, *l_range)
            Wd = W.log_uniform_int(rng, *w_range)
            e = W.layered_dag(L, Wd, seed * 1_000_003 + i)
            reqs.append(Request(i, "tc", (e,), L * Wd, float(t[i])))
        else:
            scale = int(rng.integers(min_scale, max_scale + 1))
            nodes = 1 << scale
            e = W.rmat_edges(scale, 4 * nodes, seed=seed * 1_000_003 + i)
            reqs.append(Request(i, "sg", (e,), nodes, float(t[i])))
    for r in reqs:
        r.est_bytes, r.est_tuples = hbm_estimate(r)
    return reqs


def hbm_estimate(r: Request) -> tuple[int, int]:
    """(bytes a query needs on the device, candidates of its first join);
    see the module docstring."""
    n = r.nodes
    e = r.inputs[0]
    bitmap = (n * max(32, 1 << int(np.ceil(np.log2(max(n, 32) / 32)) + 5))) // 8
    outdeg = np.bincount(e[:, 0].astype(np.int64), minlength=n)
    indeg = np.bincount(e[:, 1].astype(np.int64), minlength=n)
    if r.kind == "tc":
        # first join: path DELTA (= edges) probes edge_rev on its c0 (= y)
        cands = int((indeg * outdeg).sum())
        bitmaps = 3
    else:
        # init join: edge x edge on the shared source
        cands = int((outdeg.astype(np.int64) ** 2).sum())
        bitmaps = 4
    return bitmaps * bitmap + 16 * (cands + len(e)), cands + len(e)


def device_estimate(eng: Engine, r: Request) -> tuple[int, int]:
    """hbm_estimate with the first join's candidates from its count pass on
    the device: the relations that join reads, loaded as the program loads
    them (programs.tc: path(x, y) probes edge reversed on y; programs.sg:
    edge joined with itself on the source), then gdl_join_count."""
    n = r.nodes
    e = r.inputs[0]
    bitmap = (n * max(32, 1 << int(np.ceil(np.log2(max(n, 32) / 32)) + 5))) // 8
    eng.clear()
    if r.kind == "tc":
        edge_rev = eng.relation("edge_2__2_1")
        path = eng.relation("path_2__1_2", index_flag=False)
        eng.load(path, e)
        eng.load(edge_rev, W.reverse(e))
        # the first iteration's DELTA of path is its FULL (src/lie.cu:49-59)
        cands = eng.join_count(edge_rev, FULL, path, FULL)
        bitmaps = 3
    else:
        edge = eng.relation("edge_2__1_2")
        eng.load(edge, e)
        cands = eng.join_count(edge, FULL, edge, FULL)
        bitmaps = 4
    return bitmaps * bitmap + 16 * (cands + len(e)), cands + len(e)


def percentiles(lat):
    if not lat:
        return {"p50_ms": None, "p99_ms": None, "mean_ms": None}
    a = np.sort(np.asarray(lat)) * 1e3
    return {"p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)),
            "mean_ms": float(a.mean())}


class Server:
    def __init__(self, slots=2, budget_bytes=24 << 30, max_batch=256, batched=True, device=0,
                 tuple_cap=1 << 29, plain_min_nodes=1 << 12, device_admission=True):
        self.slots = slots
        self.device_admission = device_admission and batched
        self.plain_min_nodes = plain_min_nodes
        self.budget = budget_bytes
        self.tuple_cap = tuple_cap
        self.max_batch = max_batch
        self.batched = batched
        self.device = device
        self.queue = collections.deque()
        self.cv = threading.Condition()
        self.done = False
        self.batches = []  # (kind, size, seconds)
        self.splits = 0    # batches split after the engine refused their size
        self.error = None

    def _take(self):
        """Next batch: the oldest waiting query's kind, then every waiting
        query of that kind, in arrival order, within budget and max_batch."""
        if not self.queue:
            return []
        kind = self.queue[0].kind
        if not self.batched or self._alone(self.queue[0]):
            return [self.queue.popleft()]
        take, used, tuples, keep = [], 0, 0, collections.deque()
        while self.queue:
            r = self.queue.popleft()
            if (r.kind == kind and not self._alone(r) and len(take) < self.max_batch
                    and (not take or (used + r.est_bytes <= self.budget
                                      and tuples + r.est_tuples <= self.tuple_cap))):
                take.append(r)
                used += r.est_bytes
                tuples += r.est_tuples
            else:
                keep.append(r)
        self.queue = keep
        return take

    def _alone(self, r) -> bool:
        """Served alone through the plain engine (see the module docstring)."""
        return bool(self.plain_min_nodes) and r.nodes >= self.plain_min_nodes

    def _worker(self, t0):
        try:
            self._work(t0)
        except BaseException as exc:  # surfaced by serve()
            with self.cv:
                self.error = exc
                self.done = True
                self.queue.clear()
                self.cv.notify_all()

    def _work(self, t0):
        eng = Engine("gpu", device=self.device)
        try:
            while True:
                with self.cv:
                    while not self.queue and not self.done:
                        self.cv.wait()
                    if not self.queue and self.done:
                        return
                    reqs = self._take()
                now = time.perf_counter() - t0
                for r in reqs:
                    r.start = now
                prog = PROGRAMS[reqs[0].kind]
                ts = time.perf_counter()
                results = self._run(eng, prog, reqs)
                end = time.perf_counter() - t0
                self.batches.append((reqs[0].kind, len(reqs), time.perf_counter() - ts))
                for r, res in zip(reqs, results):
                    r.result = res
                    r.finish = end
        finally:
            eng.close()

    def _run(self, eng, prog, reqs) -> list:
        """Results of one batch (or, unbatched, of each query in turn); a
        batch refused for its size is split in halves."""
        if not self.batched or len(reqs) == 1:
            return B.run_plain_loop(eng, prog, [r.inputs for r in reqs]).results
        try:
            return B.run_batched(eng, prog, [r.inputs for r in reqs],
                                 node_counts=[r.nodes for r in reqs]).results
        except GdlError as exc:
            if exc.code not in _TOO_LARGE or len(reqs) == 1:
                raise
            self.splits += 1  # run_batched clears the engine before each half
            h = len(reqs) // 2
            return self._run(eng, prog, reqs[:h]) + self._run(eng, prog, reqs[h:])

    def serve(self, requests, time_scale=1.0):
        """Release requests at their arrival times (scaled) and serve them.
        Each request's HBM estimate is taken on arrival from its first
        join's count pass (device_estimate) when `device_admission`."""
        t0 = time.perf_counter()
        workers = [threading.Thread(target=self._worker, args=(t0,)) for _ in range(self.slots)]
        est = Engine("gpu", device=self.device) if self.device_admission else None
        for w in workers:
            w.start()
        try:
            for r in requests:
                delay = r.arrival * time_scale - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                r.arrival = r.arrival * time_scale
                if est is not None and not self._alone(r):
                    # (a query served alone is admitted whatever its size)
                    r.est_bytes, r.est_tuples = device_estimate(est, r)
                with self.cv:
                    if self.error is not None:
                        break
                    self.queue.append(r)
                    self.cv.notify()
        finally:
            if est is not None:
                est.close()
        with self.cv:
            self.done = True
            self.cv.notify_all()
        for w in workers:
            w.join()
        if self.error is not None:
            raise RuntimeError(f"serving failed: {self.error!r}") from self.error
        makespan = max(r.finish for r in requests)
        lat = [r.finish - r.arrival for r in requests]
        out = {"requests": len(requests), "makespan_s": makespan,
               "throughput_rps": len(requests) / makespan, "batches": len(self.batches),
               "mean_batch": float(np.mean([b[1] for b in self.batches])) if self.batches else 0,
               "splits": self.splits}
        out.update(percentiles(lat))
        for kind in ("tc", "sg"):
            sub = [r.finish - r.arrival for r in requests if r.kind == kind]
            if sub:
                out[kind] = percentiles(sub)
        return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--slots", type=int, default=2)
    ap.add_argument("--budget-gb", type=float, default=24.0)
    ap.add_argument("--max-scale", type=int, default=14)
    ap.add_argument("--plain", action="store_true", help="serve one query at a time, unbatched")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--plain-min-scale", type=int, default=12,
                    help="SG queries on 2^this nodes or more run alone, unbatched (0: never)")
    a = ap.parse_args()
    reqs = make_stream(a.requests, a.rate, seed=a.seed, max_scale=a.max_scale)
    srv = Server(slots=1 if a.plain else a.slots, budget_bytes=int(a.budget_gb * (1 << 30)),
                 batched=not a.plain,
                 plain_min_nodes=(1 << a.plain_min_scale) if a.plain_min_scale else 0)
    stats = srv.serve(reqs)
    stats.update({"mode": "plain" if a.plain else "batched", "rate": a.rate,
                  "slots": srv.slots})
    print(json.dumps(stats), flush=True)


if __name__ == "__main__":
    main()
