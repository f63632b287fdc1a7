"""Autotuner for the fixpoint engine's launch and layout parameters.

The reference fixes its launch shape per driver (grid = 32 x SMs, block 512,
test/tc.cu:223-225) and its index load factor (0.8, src/relation.cu:836).
Here the engine exposes, through gdl_tuning, the choices whose best value
depends on the instance: the dedup path (bitmaps or radix sort + merge), the
largest domain kept as bitmaps, the form of a join into bitmaps (one
probe-and-expand pass, or count + materialise passes), the CTAs per SM of
the join's count and materialisation passes, the slots per key of the
hashed index (its load factor), the block size of the one-pass join, the
radix sort's digit width (6, 8 or 10 bits; the number of passes follows
the key width) and the join tile of the row-gather form (in-edges per unit
of work).

The tuner buckets a workload by program and by log2 of its node and tuple
counts.  It times every combination of SPACE on the workload (device time
of the fixpoints, best of `reps`), then, from the fastest, tries each value
of every REFINE parameter in turn and keeps what is faster (coordinate
descent), and remembers the result per (GPU, bucket) in a JSON cache.
Results never depend on the choice: every configuration gives the same
tuples, sizes and loop-pass counts.
"""
from __future__ import annotations

import itertools
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_CACHE = os.path.join(HERE, "tuning_cache.json")

# Candidate values per parameter (0 keeps the engine's default).
SPACE = {
    "dedup": ["dense", "sort"],
    "dense_join_passes": [1, 2],
    "join_aggregate": [1, 2],
    "join_ctas_per_sm": [4, 8, 16],
    "count_ctas_per_sm": [2, 4, 8],
    "index_slots_per_key": [2, 4],
    "pull_joins": [2, 1],
}
# Tried one at a time from the best of SPACE (default first).
REFINE = {
    "join_block": [256, 128, 512],
    "radix_bits": [8, 6, 10],
    "rows_piece": [32, 16, 8],
}


def _redundant(cfg: dict) -> bool:
    """Configurations that differ from an earlier one only in a parameter
    their path does not read: the join form and bit aggregation of the sort
    path, the aggregation of the two-pass dense join, and the grids of the
    count / materialise passes of the one-pass dense join, and the pull
    form's switch on the sort path."""
    one_pass = cfg.get("dense_join_passes", 1) == 1
    if cfg.get("dedup") == "sort" and (not one_pass or cfg.get("join_aggregate", 1) != 1 or
                                       cfg.get("pull_joins", 2) != 2):
        return True
    if cfg.get("dedup") == "dense" and one_pass:
        return (cfg.get("count_ctas_per_sm", 2) != 2 or cfg.get("join_ctas_per_sm", 4) != 4)
    if cfg.get("dedup") == "dense" and cfg.get("join_aggregate", 1) != 1:
        return True
    return False


def bucket(program: str, inputs) -> str:
    """Size class of a workload: program, log2(nodes), log2(tuples)."""
    n_rows = sum(len(x) for x in inputs)
    nodes = 1
    for x in inputs:
        if len(x):
            nodes = max(nodes, int(np.asarray(x).max()) + 1)
    return f"{program}:n{int(math.log2(max(nodes, 1)))}:t{int(math.log2(max(n_rows, 1)))}"


def candidates(space=SPACE, limit=None):
    keys = list(space)
    out = [dict(zip(keys, vals)) for vals in itertools.product(*(space[k] for k in keys))]
    out = [c for c in out if not _redundant(c)]
    return out[:limit] if limit else out


def measure(eng, prog, inputs, cfg, reps=2) -> float:
    """Best device milliseconds of the program's fixpoints under cfg."""
    def run(e):
        e.clear()
        r = prog(e, *inputs, sync=e.sync)
        return sum(lie.stats()["ms"] for lie in r.lies.values())
    return measure_runner(eng, run, cfg, reps)


def measure_runner(eng, run, cfg, reps=2) -> float:
    """Best of `reps` calls of run(eng) -> device milliseconds under cfg; a
    configuration the engine refuses for the workload (a status such as the
    list limit) scores as infinitely slow, and the engine is cleared."""
    from gdlog_b200 import GdlError
    eng.set_tuning(**cfg)
    try:
        return min(run(eng) for _ in range(reps))
    except GdlError:
        eng.clear()
        return math.inf


def batch_bucket(program: str, instances) -> str:
    """Size class of a batch of instances: program, instance count (log2),
    largest instance (log2 nodes), total tuples (log2)."""
    n_rows = sum(len(x) for inp in instances for x in inp)
    nodes = 1
    for inp in instances:
        for x in inp:
            if len(x):
                nodes = max(nodes, int(np.asarray(x).max()) + 1)
    return (f"{program}-batch:i{int(math.log2(max(len(instances), 1)))}"
            f":n{int(math.log2(nodes))}:t{int(math.log2(max(n_rows, 1)))}")


class Tuner:
    def __init__(self, cache_path: str = DEFAULT_CACHE, gpu_name: str = "B200"):
        self.path = cache_path
        self.gpu = gpu_name
        self.cache = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def key(self, program: str, inputs) -> str:
        return f"{self.gpu}|{bucket(program, inputs)}"

    def lookup(self, program: str, inputs):
        return self.cache.get(self.key(program, inputs))

    def tune(self, eng, prog, inputs, space=SPACE, reps=2, save=True) -> dict:
        """Time every candidate on this workload; remember and return the best."""
        def run(e):
            e.clear()
            r = prog(e, *inputs, sync=e.sync)
            return sum(lie.stats()["ms"] for lie in r.lies.values())
        return self.tune_runner(eng, self.key(prog.__name__, inputs), run, space, reps, save)

    def tune_runner(self, eng, key: str, run, space=SPACE, reps=2, save=True,
                    refine=None) -> dict:
        """tune() for any run(eng) -> device milliseconds (e.g. a batched
        fixpoint over many instances), cached under `key`.  `refine`
        (default REFINE when `space` is SPACE, else none): parameters tried
        one at a time from the best of `space`."""
        if refine is None:
            refine = REFINE if space is SPACE else {}
        defaults = {k: v[0] for k, v in refine.items()}
        results = []
        for cfg in candidates(space):
            cfg = {**cfg, **defaults}
            results.append((measure_runner(eng, run, cfg, reps), cfg))
        results.sort(key=lambda x: x[0])
        best_ms, best = results[0]
        first = {**candidates(space)[0], **defaults}
        default_ms = next((ms for ms, c in results if c == first), None)
        tried = len(results)
        for name, values in refine.items():
            for v in values[1:]:
                cfg = {**best, name: v}
                ms = measure_runner(eng, run, cfg, reps)
                tried += 1
                if ms < best_ms:
                    best_ms, best = ms, cfg
        rec = {"config": best, "ms": best_ms, "default_ms": default_ms, "tried": tried}
        self.cache[key] = rec
        if save:
            with open(self.path, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
        eng.set_tuning(**best)
        return rec

    def apply_key(self, eng, key: str) -> dict | None:
        """Set the cached best configuration stored under `key`, if any."""
        rec = self.cache.get(key)
        if rec:
            eng.set_tuning(**rec["config"])
        return rec

    def apply(self, eng, prog, inputs) -> dict | None:
        """Set the cached best configuration for this workload, if any."""
        rec = self.lookup(prog.__name__, inputs)
        if rec:
            eng.set_tuning(**rec["config"])
        return rec
