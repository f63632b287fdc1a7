"""load_relation's sort + unique (src/relation.cu:523-632): the radix sort
with merge-path dedup and the domain-bitmap listing (gdl_tuning.load_dedup
1 and 2) give the same FULL as numpy's sorted unique rows, around the
bitmap path's limits (more than 4096 rows; ids below 2^15), and a program
run on either gives the same answers."""
import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import DELTA, FULL, Engine

pytestmark = pytest.mark.gpu


def _rows(n, maxv, seed):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, maxv, size=(n, 2), dtype=np.uint64)
    # repeats, in load order far apart
    if n > 8:
        r[n // 2:n // 2 + n // 8] = r[:n // 8]
    return r


def _unique(rows):
    return np.unique(rows, axis=0)


@pytest.mark.parametrize("n,maxv", [(4096, 1 << 14), (4097, 1 << 14), (5000, 200),
                                    (40000, 1 << 14), (200000, 1 << 15), (120000, 1 << 12),
                                    (70000, (1 << 15) + 1), (10000, 1 << 20)])
def test_load_paths_equal_numpy(n, maxv):
    rows = _rows(n, maxv, seed=n ^ maxv)
    want = _unique(rows)
    for mode in (1, 2):
        with Engine("gpu") as g:
            g.set_tuning(load_dedup=mode)
            r = g.relation("r")
            g.load(r, rows)
            got = r.rows(FULL)
            assert r.size(FULL) == len(want)
            assert np.array_equal(got, want), mode
            assert r.size(DELTA) == 0


def test_reload_and_mixed_widths():
    """Loads after wider ones (the domain grows with the largest id seen),
    a reload replacing FULL, and an empty load, on the bitmap path."""
    with Engine("gpu") as g:
        assert g.get_tuning().load_dedup == 2
        a, b = g.relation("a"), g.relation("b")
        ra = _rows(9000, 1 << 10, 1)
        g.load(a, ra)
        rb = _rows(30000, 1 << 14, 2)
        g.load(b, rb)
        assert np.array_equal(a.rows(FULL), _unique(ra))
        assert np.array_equal(b.rows(FULL), _unique(rb))
        ra2 = _rows(50000, 1 << 13, 3)
        g.load(a, ra2)
        assert np.array_equal(a.rows(FULL), _unique(ra2))
        g.load(b, None)
        assert b.size(FULL) == 0


@pytest.mark.parametrize("prog,make", [
    ("sg", lambda: (W.rmat_edges(12, 8000, seed=3),)),
    ("tc", lambda: (W.grid_edges(32, 32),)),
])
def test_programs_equal_on_both_load_paths(prog, make):
    """The raw load order (DELTA at LIE start, src/lie.cu:49-59) is kept
    apart from FULL, so fixpoints over either load path agree, traces
    included."""
    inputs = make()
    out = []
    for mode in (1, 2):
        with Engine("gpu") as g:
            g.set_tuning(load_dedup=mode)
            r = getattr(P, prog)(g, *inputs)
            out.append(({k: (v.size(), v.digest()) for k, v in r.relations.items()},
                        dict(r.iterations),
                        {k: lie.trace().tolist() for k, lie in r.lies.items()}))
    assert out[0] == out[1]
