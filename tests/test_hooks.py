"""Program hooks that are not column selections, through the drop-in C++
API (tests/cpp/compat_drivers.cu).

The reference calls a program's __device__ hooks through function pointers
for every candidate tuple (src/relation.cu:290-403).  The drop-in probes a
hook on 256 randomised samples and hands it to the engine as a column
selection only if it is one on all of them; anything else must run through
its function pointer and give the exact answer.  Checked here:

  * a generator that compares columns, max(inner[1], outer[1]); a predicate
    t[0] != t[1] && t[0] < 100 (agrees with != on most tuples); copy and
    ACopy hooks that flip a bit -- each against a CPU restatement of the
    same program (below), sizes, digests and loop passes;
  * that each is classified as the probe should (GDLOG_HOOK_LOG);
  * the reference programs (TC, SG, CSPA) with every hook forced through
    its function pointer (GDLOG_EXACT_HOOKS=1) against the golden answers.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import workloads as W
from gdlog_b200 import digest_rows
from test_oracle import GOLDEN, build_workload

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVERS = os.path.join(REPO, "gdlog-multinode_b200", "lib", "compat_drivers")


# -- CPU restatement of a LIE (src/lie.cu:26-274) over Python sets ----------

class Rel:
    def __init__(self, rows=()):
        self.full = set(map(tuple, rows))
        self.delta = set()
        self.newt = set()


def run_lie(update, ops, tmps=()):
    """ops: ("join", inner, inner_ver, outer, outer_ver, out, gen, pred),
    ("copy", src, src_ver, dest, hook), ("acopy", src, dest, hook).
    Inputs here repeat no row, so DELTA starts as FULL (src/lie.cu:49-59)."""
    for r in update:
        r.delta = set(r.full)
    copied = set()
    it = 0
    while True:
        for i, op in enumerate(ops):
            if op[0] == "join":
                _, inner, iv, outer, ov, out, gen, pred = op
                ins = inner.delta if iv == "delta" else inner.full
                outs = {"delta": outer.delta, "full": outer.full, "newt": outer.newt}[ov]
                if not outs or not ins:  # src/join.cu:38-45 (no empty inner here)
                    continue
                by_key = {}
                for t in ins:
                    by_key.setdefault(t[0], []).append(t)
                for o in list(outs):
                    for t in by_key.get(o[0], ()):
                        res = gen(t, o)
                        if pred is None or pred(res):
                            out.newt.add(res)
            elif op[0] == "copy":
                _, src, sv, dest, hook = op
                if sv == "full":
                    if i in copied:
                        continue
                    copied.add(i)
                s = src.full if sv == "full" else src.delta
                if not s:  # src/copy.cu:24-27
                    dest.newt = set()
                    continue
                dest.newt |= {hook(t) for t in s}
            else:
                _, src, dest, hook = op
                dest.newt = {hook(t) for t in src.newt}
        for r in tmps:
            r.newt = set()
        done = True
        for r in update:
            if not r.newt:
                r.delta = set()
                continue
            r.delta = r.newt - r.full
            r.full |= r.delta
            r.newt = set()
            done = done and not r.delta
        it += 1
        if done:
            return it


def summary(rel):
    rows = np.array(sorted(rel.full), dtype=np.uint64).reshape(-1, 2)
    return len(rows), hex(digest_rows(rows))


def swap(rows):
    return [(b, a) for a, b in rows]


def cpu_hook_max(e):
    edge, path = Rel(swap(e)), Rel(e)
    it = run_lie([path], [("join", edge, "full", path, "delta", path,
                           lambda i, o: (max(i[1], o[1]), o[1]), None)])
    return {"sizes": {"path": summary(path)[0]}, "digests": {"path": summary(path)[1]},
            "iterations": {"lie": it}}


def cpu_hook_pred(e):
    pred = lambda t: t[0] != t[1] and t[0] < 100  # noqa: E731
    edge, sg, tmp = Rel(e), Rel(), Rel()
    it0 = run_lie([sg], [("join", edge, "full", edge, "full", sg,
                          lambda i, o: (i[1], o[1]), pred)])
    it1 = run_lie([sg], [("join", edge, "full", sg, "delta", tmp, lambda i, o: (o[1], i[1]), None),
                         ("join", edge, "full", tmp, "newt", sg, lambda i, o: (o[1], i[1]), pred)],
                  tmps=[tmp])
    return {"sizes": {"sg": summary(sg)[0]}, "digests": {"sg": summary(sg)[1]},
            "iterations": {"init": it0, "lie": it1}}


def cpu_hook_copy(e):
    edge, r, m, d = Rel(swap(e)), Rel(), Rel(), Rel()
    xor = lambda t: (t[1], t[0] ^ 1)  # noqa: E731
    swap_xor = lambda t: (t[1] ^ 1, t[0])  # noqa: E731
    it = run_lie([r, m, d], [("copy", edge, "full", r, xor),
                             ("join", edge, "full", r, "delta", r, lambda i, o: (i[1], o[1]), None),
                             ("copy", r, "delta", d, xor),
                             ("acopy", r, m, swap_xor)])
    out = {"sizes": {}, "digests": {}, "iterations": {"lie": it}}
    for name, rel in (("r", r), ("m", m), ("d", d)):
        out["sizes"][name], out["digests"][name] = summary(rel)
    return out


CASES = {
    "hook_max": (cpu_hook_max, lambda: W.rmat_edges(7, 300, seed=21)),
    "hook_pred": (cpu_hook_pred, lambda: W.rmat_edges(8, 700, seed=22)),
    "hook_copy": (cpu_hook_copy, lambda: W.rmat_edges(6, 150, seed=23)),
}


def test_cpu_restatement_matches_oracle():
    """The restatement above gives the oracle's answers on plain programs:
    TC, and SG (its tmp relation read as NEWT, a predicate)."""
    import programs as P
    from gdlog_b200 import Engine
    e = W.grid_edges(8, 8)
    edge, path = Rel(swap(e)), Rel(e)
    it = run_lie([path], [("join", edge, "full", path, "delta", path,
                           lambda i, o: (i[1], o[1]), None)])
    with Engine("oracle") as o:
        r = P.tc(o, e)
        assert (len(path.full), summary(path)[1], it) == (
            r.output.size(), hex(r.output.digest()), r.iterations["tc"])
    e = W.rmat_edges(7, 400, seed=5)
    edge, sg, tmp = Rel(e), Rel(), Rel()
    ne = lambda t: t[0] != t[1]  # noqa: E731
    it0 = run_lie([sg], [("join", edge, "full", edge, "full", sg, lambda i, o: (i[1], o[1]), ne)])
    it1 = run_lie([sg], [("join", edge, "full", sg, "delta", tmp, lambda i, o: (o[1], i[1]), None),
                         ("join", edge, "full", tmp, "newt", sg, lambda i, o: (o[1], i[1]), None)],
                  tmps=[tmp])
    with Engine("oracle") as o:
        r = P.sg(o, e)
        assert (len(sg.full), summary(sg)[1], it0, it1) == (
            r.output.size(), hex(r.output.digest()), r.iterations["init"], r.iterations["sg"])


def run_driver(prog, files, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    r = subprocess.run([DRIVERS, prog, *files], capture_output=True, text=True, timeout=600,
                       env=env)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):]), r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("prog", sorted(CASES))
def test_non_selection_hooks_run_exactly(tmp_path, prog):
    cpu, make = CASES[prog]
    e = make()
    p = tmp_path / "e.tsv"
    W.write_tsv(str(p), e)
    got, log = run_driver(prog, [str(p)], {"GDLOG_HOOK_LOG": "1"})
    want = cpu([tuple(map(int, r)) for r in e.tolist()])
    assert got == want
    assert "device function pointers" in log


@pytest.mark.gpu
def test_probe_classification(tmp_path):
    """Selections go to the engine's own kernels; max() and the compound
    predicate do not."""
    e = W.rmat_edges(6, 150, seed=3)
    p = tmp_path / "e.tsv"
    W.write_tsv(str(p), e)
    _, log = run_driver("sg", [str(p)], {"GDLOG_HOOK_LOG": "1"})
    assert "device function pointers" not in log
    assert log.count("RelationalJoin hooks -> column selection") == 3
    _, log = run_driver("hook_max", [str(p)], {"GDLOG_HOOK_LOG": "1"})
    assert "RelationalJoin hooks -> device function pointers" in log
    _, log = run_driver("hook_pred", [str(p)], {"GDLOG_HOOK_LOG": "1"})
    lines = [ln for ln in log.splitlines() if "RelationalJoin" in ln]
    # init join (predicate), tmp join (plain), sg join (predicate)
    assert lines == ["gdlog: RelationalJoin hooks -> device function pointers",
                     "gdlog: RelationalJoin hooks -> column selection",
                     "gdlog: RelationalJoin hooks -> device function pointers"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tc_grid_16x16", "tc_dag_L12_W10_s2", "sg_rmat_s8_600_s1",
                                  "cspa_v120_s1"])
def test_reference_programs_through_function_pointers(tmp_path, name):
    """Every hook of TC, SG and CSPA run through its function pointer
    (joins with and without predicate, FULL copies run once, DELTA copies,
    ACopy, tmp relations): the golden answers."""
    prog, args = build_workload(name)
    files = []
    for i, rows in enumerate(args):
        f = tmp_path / f"in{i}.tsv"
        W.write_tsv(str(f), rows)
        files.append(str(f))
    got, log = run_driver(prog.__name__, files, {"GDLOG_EXACT_HOOKS": "1",
                                                  "GDLOG_HOOK_LOG": "1"})
    assert "column selection" not in log
    want = GOLDEN["workloads"][name]
    assert got["sizes"] == want["sizes"]
    assert got["iterations"] == want["iterations"]
    assert got["digests"] == want["digests"]
