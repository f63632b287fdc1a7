"""Failure handling without a GPU fault.

A bounded device-side wait that runs out makes the call return
GDL_E_TIMEOUT and leaves the CUDA context usable: the test makes one run
out on purpose (gdl_engine_test_timeout: the next fixpoint's first control
kernel waits on a device flag that nothing sets), checks the status, that
the engine then refuses work, and that gdl_engine_clear recovers it so the
next programs give the oracle's answers.  With the look-back waits cut to a
couple of polls (gdl_tuning.spin_limit_log2) a run is either right or
reports the timeout, never wrong."""
import pytest

import programs as P
import workloads as W
from gdlog_b200 import Engine, GdlError

pytestmark = pytest.mark.gpu

GDL_E_TIMEOUT = 5


def answer(r):
    return (r.output.size(), dict(r.iterations), r.output.digest())


def test_timeout_is_reported_and_clear_recovers():
    e = W.grid_edges(12, 12)
    s = W.rmat_edges(12, 6000, seed=12)
    with Engine("oracle") as o:
        want_tc = answer(P.tc(o, e))
        want_sg = answer(P.sg(o, s))
    with Engine("gpu") as g:
        g.test_timeout(1000)
        with pytest.raises(GdlError) as err:
            P.tc(g, e, sync=g.sync)
        assert err.value.code == GDL_E_TIMEOUT
        # further work is refused until the engine is cleared
        x = g.relation("x")
        with pytest.raises(GdlError):
            g.load(x, e)
        g.clear()
        assert answer(P.tc(g, e, sync=g.sync)) == want_tc
        g.clear()
        assert answer(P.sg(g, s, sync=g.sync)) == want_sg
        # a timeout in the middle of a program: its second LIE
        g.clear()
        edge = g.relation("edge")
        path = g.relation("path", index_flag=False)
        g.load(edge, W.reverse(e))
        g.load(path, e)
        lie = g.lie()
        lie.add_relations(edge, True)
        lie.add_relations(path, False)
        lie.add_join(edge, 1, path, 0, path, P.REORDER_PATH)
        lie.max_iteration = 3
        lie.fixpoint()
        g.test_timeout(10)
        lie2 = g.lie()
        lie2.add_relations(edge, True)
        lie2.add_relations(path, False)
        lie2.add_join(edge, 1, path, 0, path, P.REORDER_PATH)
        with pytest.raises(GdlError) as err:
            lie2.fixpoint()
        assert err.value.code == GDL_E_TIMEOUT
        g.clear()
        assert answer(P.tc(g, e, sync=g.sync)) == want_tc


@pytest.mark.parametrize("mode", ["sort", "dense"])
def test_tiny_wait_limit_is_never_wrong(mode):
    """Look-back waits cut to 2 polls: every run is the oracle's answer or a
    reported timeout; after clear() and the default limit, the answer."""
    s = W.rmat_edges(12, 6000, seed=7)
    with Engine("oracle") as o:
        want = answer(P.sg(o, s))
    outcomes = []
    with Engine("gpu", dedup=mode) as g:
        default = g.get_tuning().spin_limit_log2
        g.set_tuning(spin_limit_log2=1)
        for _ in range(3):
            try:
                got = answer(P.sg(g, s, sync=g.sync))
                assert got == want
                outcomes.append("ok")
                g.clear()
            except GdlError as exc:
                assert exc.code == GDL_E_TIMEOUT
                outcomes.append("timeout")
                g.clear()
        g.set_tuning(spin_limit_log2=default)
        assert answer(P.sg(g, s, sync=g.sync)) == want
    assert len(outcomes) == 3
