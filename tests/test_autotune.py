"""Autotuner (autotune.py): every tuning configuration gives bit-identical
results, the tuner picks the fastest and remembers it per size bucket."""
import json

import pytest

import autotune as A
import programs as P
import workloads as W
from gdlog_b200 import Engine, GdlError


def test_bucket_and_candidates():
    e = W.grid_edges(16, 16)
    assert A.bucket("tc", (e,)) == "tc:n8:t8"
    cands = A.candidates()
    # sort: 3 x 3 x 2 grids; dense with 2 passes: the same, push or pull
    # form; dense with one pass: the index choice and the bit aggregation,
    # push or pull form
    assert len(cands) == 18 + 2 * 18 + 2 * 4
    assert {c["dedup"] for c in cands} == {"dense", "sort"}
    assert {c["dense_join_passes"] for c in cands} == {1, 2}
    assert {c["pull_joins"] for c in cands} == {1, 2}


@pytest.mark.gpu
def test_tuning_values_validated():
    with Engine("gpu") as g:
        with pytest.raises(GdlError):
            g.set_tuning(index_slots_per_key=3)
        with pytest.raises(GdlError):
            g.set_tuning(dense_max_bits=40)
        g.set_tuning(join_ctas_per_sm=16, dedup="sort")
        t = g.get_tuning().as_dict()
        assert t["join_ctas_per_sm"] == 16 and t["dedup"] == 1


@pytest.mark.gpu
def test_every_configuration_gives_the_same_result(tmp_path):
    e = W.rmat_edges(8, 600, seed=2)
    outs = set()
    with Engine("gpu") as g:
        for cfg in A.candidates():
            g.set_tuning(**cfg)
            g.clear()
            r = P.sg(g, e, sync=g.sync)
            outs.add((r.output.size(), r.output.digest(), tuple(sorted(r.iterations.items()))))
        assert len(outs) == 1
        tuner = A.Tuner(str(tmp_path / "cache.json"))
        rec = tuner.tune(g, P.sg, (e,), space={"dedup": ["dense", "sort"],
                                               "join_ctas_per_sm": [4, 8]}, reps=1)
        assert rec["ms"] <= min(rec["default_ms"], rec["ms"]) + 1e-9
        assert json.load(open(tmp_path / "cache.json"))
        assert A.Tuner(str(tmp_path / "cache.json")).lookup("sg", (e,))["config"] == rec["config"]
