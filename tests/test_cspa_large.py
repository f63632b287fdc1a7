"""GPU parity of the points-to analysis (test/cspa.cu:100-379) at sizes the
list oracle cannot finish, against the bit-matrix oracle's committed answers
(tests/golden/cspa_large.json, written by tests/golden/make_cspa_large.py):
sizes, loop-pass counts, digests of the sorted results and the whole
per-iteration (dedup, delta, full) log of src/lie.cu:193-197, bit-exact.

cspa_c3 is the 20,000-variable configuration (40,000 assign and 15,000
dereference pairs, source bounded Zipf(1.1), target uniform, seed 3):
value_flow 87,066,231, memory_alias 109,683,540 and value_alias 359,257,336
tuples after 3 + 12 loop passes.  It runs with the joins gathered by output
row (the default) and with every join pushed, one reduction per candidate.
"""
import json
import os

import pytest

import programs as P
from gdlog_b200 import Engine

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LARGE = json.load(open(os.path.join(HERE, "golden", "cspa_large.json")))


def summarize(r):
    return {
        "sizes": {k: v.size() for k, v in r.relations.items()},
        "digests": {k: hex(v.digest()) for k, v in r.relations.items()},
        "iterations": dict(r.iterations),
        "traces": {k: lie.trace().tolist() for k, lie in r.lies.items()},
    }


def check(name, mode):
    from golden.make_cspa_large import WORKLOADS
    with Engine("gpu", dedup=mode) as g:
        got = summarize(P.cspa(g, *WORKLOADS[name](), sync=g.sync))
    want = LARGE[name]
    assert got["sizes"] == want["sizes"]
    assert got["iterations"] == want["iterations"]
    assert got["digests"] == want["digests"]
    assert got["traces"] == want["traces"]


@pytest.mark.parametrize("mode", ["dense", "dense_push", "dense_2pass"])
def test_cspa_2000_vars(mode):
    check("cspa_v2000_s3", mode)


def test_cspa_2000_vars_sorted_lists_refuse():
    """The sorted-list path materialises join candidates (about 48 G here,
    beyond its 2^30-row limit): it must stop with a status, not answer."""
    from golden.make_cspa_large import WORKLOADS
    from gdlog_b200 import GdlError
    with Engine("gpu", dedup="sort") as g:
        with pytest.raises(GdlError, match="UNSUPPORTED"):
            P.cspa(g, *WORKLOADS["cspa_v2000_s3"](), sync=g.sync)


@pytest.mark.parametrize("mode", ["dense", "dense_push"])
def test_cspa_6000_vars(mode):
    check("cspa_v6000_s3", mode)


@pytest.mark.parametrize("mode", ["dense", "dense_push"])
def test_cspa_c3_20000_vars(mode):
    check("cspa_c3", mode)
