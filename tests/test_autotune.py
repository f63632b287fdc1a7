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


def test_refine_parameters_start_from_the_default():
    """The block size, radix digit width and row-gather join tile are tried
    one at a time, the engine's default first."""
    assert A.REFINE["join_block"][0] == 256
    assert A.REFINE["radix_bits"][0] == 8
    assert A.REFINE["rows_piece"][0] == 32
    assert set(A.REFINE["radix_bits"]) == {6, 8, 10}


@pytest.mark.gpu
def test_tuning_values_validated():
    with Engine("gpu") as g:
        with pytest.raises(GdlError):
            g.set_tuning(index_slots_per_key=3)
        with pytest.raises(GdlError):
            g.set_tuning(dense_max_bits=40)
        for bad in ({"radix_bits": 7}, {"join_block": 64}, {"rows_piece": 64},
                    {"load_dedup": 3}):
            with pytest.raises(GdlError):
                g.set_tuning(**bad)
        g.set_tuning(join_ctas_per_sm=16, dedup="sort", radix_bits=10, join_block=512,
                     rows_piece=8, load_dedup=1)
        t = g.get_tuning().as_dict()
        assert t["join_ctas_per_sm"] == 16 and t["dedup"] == 1
        assert (t["radix_bits"], t["join_block"], t["rows_piece"]) == (10, 512, 8)
        assert t["load_dedup"] == 1


@pytest.mark.gpu
@pytest.mark.parametrize("bits", [6, 8, 10])
def test_radix_digit_widths_agree(bits):
    """The sorted-list path gives the same tuples, sizes and passes with 6-,
    8- and 10-bit digits (ids of 9 and 13 bits: odd pass counts included)."""
    for scale, n in ((9, 900), (13, 6000)):
        e = W.rmat_edges(scale, n, seed=scale)
        with Engine("oracle") as o:
            ro = P.sg(o, e)
            want = (ro.output.size(), ro.output.digest(), tuple(sorted(ro.iterations.items())))
        with Engine("gpu") as g:
            g.set_tuning(dedup="sort", radix_bits=bits)
            r = P.sg(g, e, sync=g.sync)
            assert (r.output.size(), r.output.digest(),
                    tuple(sorted(r.iterations.items()))) == want


@pytest.mark.gpu
@pytest.mark.parametrize("block,piece", [(128, 8), (512, 16), (256, 32)])
def test_join_block_and_rows_piece_agree(block, piece):
    """The one-pass join's block size and the row-gather join tile change
    no result (same generation through the push form at 2^9 ids and the
    row-gather form at 2^12)."""
    for scale, n in ((9, 900), (12, 5000)):
        e = W.rmat_edges(scale, n, seed=scale + 1)
        with Engine("oracle") as o:
            ro = P.sg(o, e)
            want = (ro.output.size(), ro.output.digest(), tuple(sorted(ro.iterations.items())))
        with Engine("gpu") as g:
            g.set_tuning(join_block=block, rows_piece=piece)
            r = P.sg(g, e, sync=g.sync)
            assert (r.output.size(), r.output.digest(),
                    tuple(sorted(r.iterations.items()))) == want


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


def test_refused_configuration_scores_infinite(tmp_path):
    """A configuration the engine refuses (a GdlError from the run) loses
    instead of aborting the tune, and the engine is cleared after it."""
    from gdlog_b200 import GdlError

    class Fake:
        def __init__(self):
            self.cfg, self.cleared = {}, 0

        def set_tuning(self, **kw):
            self.cfg = kw

        def clear(self):
            self.cleared += 1

    def run(e):
        if e.cfg.get("dense_join_passes") == 2:
            raise GdlError(4, "list limit")
        return 1.0 + e.cfg.get("join_ctas_per_sm", 0) / 100

    eng = Fake()
    assert A.measure_runner(eng, run, {"dense_join_passes": 2}) == float("inf")
    assert eng.cleared == 1
    t = A.Tuner(cache_path=str(tmp_path / "cache.json"))
    space = {"dense_join_passes": [2, 1], "join_ctas_per_sm": [8, 4]}
    rec = t.tune_runner(eng, "k", run, space=space, reps=1, save=False)
    assert rec["config"]["dense_join_passes"] == 1 and rec["config"]["join_ctas_per_sm"] == 4
