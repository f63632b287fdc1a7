"""Batched fixpoints: many independent instances of one program at once.

The reference runs one fixpoint per driver invocation; a workload of many
small, uneven instances (384 layered DAGs of mixed sizes, or a stream of
queries) is then a loop of single-instance runs, each paying the engine's
per-fixpoint overheads.  Here every instance's ids are moved into their own
range, (instance << S) | local, and ONE program runs over the disjoint
union.  Because every rule joins on shared values, the union's fixpoint is
the union of the instances' fixpoints, so each instance's result is exactly
what it gets alone; the engine keeps the relations as one block-diagonal
bitmap (gdl_engine_set_instances) and reports per-instance sizes, digests
and loop-pass counts.

    results = run_batched(Engine("gpu"), programs.tc, [(edges_0,), (edges_1,), ...])
    same    = run_plain_loop(Engine("gpu"), programs.tc, [(edges_0,), ...])
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class InstanceResult:
    sizes: dict = field(default_factory=dict)       # relation -> tuples
    digests: dict = field(default_factory=dict)     # relation -> digest (local ids)
    iterations: dict = field(default_factory=dict)  # LIE -> loop passes


@dataclass
class BatchRun:
    results: list
    seconds: float          # wall seconds of the program's fixpoints
    device_ms: float        # device milliseconds of the fixpoints
    kernels: int


def node_count(inputs) -> int:
    """Local node ids used by one instance's input relations (max id + 1)."""
    m = 0
    for rows in inputs:
        if len(rows):
            m = max(m, int(np.asarray(rows).max()) + 1)
    return max(m, 1)


def globalize(instances, shift: int):
    """Concatenate the instances' input relations with ids moved to
    (instance << shift) | local.  instances: list of tuples of (n, 2) arrays,
    every instance with the same number of relations."""
    k = len(instances[0])
    out = []
    for j in range(k):
        parts = []
        for i, inp in enumerate(instances):
            rows = np.asarray(inp[j], dtype=np.uint64)
            if len(rows):
                parts.append(rows | np.uint64(i << shift))
        out.append(np.concatenate(parts) if parts else np.zeros((0, 2), dtype=np.uint64))
    return out


def shard_instances(costs, world: int, rank: int) -> list:
    """Instances of `rank` when `world` GPUs share a batch: largest cost
    first, each to the currently least-loaded rank (LPT).  Deterministic, so
    every rank computes the same partition without communicating."""
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def run_batched(eng, prog, instances, node_counts=None) -> BatchRun:
    """Run `prog` (a programs.* builder) once over all instances."""
    n = len(instances)
    counts = node_counts if node_counts is not None else [node_count(x) for x in instances]
    eng.clear()
    shift = eng.set_instances(counts)
    inputs = globalize(instances, shift)
    t0 = time.perf_counter()
    r = prog(eng, *inputs, sync=eng.sync)
    secs = time.perf_counter() - t0
    stats = {name: rel.instance_stats(n) for name, rel in r.relations.items()}
    iters = {name: lie.instance_iterations(n) for name, lie in r.lies.items()}
    lie_stats = [lie.stats() for lie in r.lies.values()]
    results = []
    for i in range(n):
        res = InstanceResult()
        for name, (sizes, digests) in stats.items():
            res.sizes[name] = int(sizes[i])
            res.digests[name] = hex(int(digests[i]))
        for name, it in iters.items():
            res.iterations[name] = int(it[i])
        results.append(res)
    eng.set_instances([])
    return BatchRun(results, secs, sum(s["ms"] for s in lie_stats),
                    sum(s["kernels"] for s in lie_stats))


def run_plain_loop(eng, prog, instances) -> BatchRun:
    """The same instances one after another through the plain engine."""
    results = []
    t0 = time.perf_counter()
    ms = 0.0
    kernels = 0
    for inp in instances:
        eng.clear()
        r = prog(eng, *inp, sync=eng.sync)
        res = InstanceResult()
        for name, rel in r.relations.items():
            res.sizes[name] = rel.size()
            res.digests[name] = hex(rel.digest())
        res.iterations = dict(r.iterations)
        results.append(res)
        if eng.kind == "gpu":
            st = [lie.stats() for lie in r.lies.values()]
            ms += sum(s["ms"] for s in st)
            kernels += sum(s["kernels"] for s in st)
    return BatchRun(results, time.perf_counter() - t0, ms, kernels)
