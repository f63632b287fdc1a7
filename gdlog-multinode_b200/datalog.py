"""Datalog rules compiled to the engine's operator program.

The reference's users write the semi-naive program by hand (test/tc.cu,
test/sg.cu, test/cspa.cu): relations in each column order a join needs
(edge_2__1_2, edge_2__2_1), one LIE per recursive component, a
RelationalJoin per rule and per recursive body atom (that atom's DELTA
against the other atoms' FULL), tmp relations for three-atom rules, and an
ACopy that keeps each swapped copy of a recursive relation current.  This
module derives that program from the rules (test/path_length.cu's too):

    path(x, y) :- edge(x, y).
    path(x, z) :- path(x, y), edge(y, z).

Supported: predicates of two columns; rule bodies of one atom (a Copy, its head any
selection of the atom's columns, e.g. vf(x, x) :- assign(x, y)), two atoms
sharing one variable (a join on it), or three atoms in a chain a-b-c (a and
b share one variable, b and c another; compiled through a tmp relation
keyed for the last join, and, for a DELTA on the third atom, through one
keyed for the first); one optional `X != Y` on the first two head
variables.
Predicates without rules are inputs (EDB).  Components of mutually
recursive predicates run as LIEs in dependency order; rules whose body has
no predicate of the component join FULL with FULL (a Copy from a FULL runs
once per LIE, src/copy.cu).

Relations of three columns join on their first (as test/path_length.cu
keys path); a head term may add a constant to a variable (l+1: GDL_PLUS) or
be a number (rows computed on the host, from a rule over one input atom).

Souffle's directives, as the reference's test/souffle/*.dl programs use
them, are read too: `.decl p(a: number, b: number)` (2 or 3 columns,
numbers; `choice-domain` over all columns but the last makes that column
dependent, as path_length's dependent_column_size 1),
`.input p(...)` (tab-separated facts: the caller's rows, else
<facts_dir>/p.facts, else the `filename` given, relative to the program),
`.output p` (<out_dir>/p.csv, sorted, tab-separated), `.printsize p`;
`_` is a fresh variable.  `python datalog.py prog.dl --facts DIR --out DIR`
runs a program file; under torchrun (WORLD_SIZE > 1) it runs with every
relation partitioned over the ranks (partition.run_file_partitioned).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np

from gdlog_b200 import DELTA, FULL, INNER, NEWT, OUTER, PLUS, PRED_NE, SRC, Engine

_TERM = r"[A-Za-z_]\w*(?:\s*\+\s*\d+)?|\d+"
_ATOM = re.compile(r"\s*([A-Za-z_]\w*)\s*\(\s*(" + _TERM + r")\s*,\s*(" + _TERM + r")\s*"
                   r"(?:,\s*(" + _TERM + r")\s*)?\)\s*")
_NE = re.compile(r"\s*([A-Za-z_]\w*)\s*!=\s*([A-Za-z_]\w*)\s*")


@dataclass(frozen=True)
class Atom:
    pred: str
    args: tuple  # terms: a variable; in a head also var+k or a number


@dataclass
class Rule:
    head: Atom
    body: list
    ne: tuple | None = None  # (X, Y): X != Y over the first two head terms
    text: str = ""


def _term(t: str):
    """(variable or None, added constant, number or None) of a term."""
    t = t.replace(" ", "")
    if t.isdigit():
        return None, 0, int(t)
    if "+" in t:
        v, k = t.split("+")
        return v, int(k), None
    return t, 0, None


@dataclass
class Directives:
    decl: dict = field(default_factory=dict)      # predicate -> arity
    dep: dict = field(default_factory=dict)       # predicate -> dependent columns (choice-domain)
    inputs: dict = field(default_factory=dict)    # predicate -> filename or None
    outputs: list = field(default_factory=list)
    printsize: list = field(default_factory=list)


_DIRECTIVE = re.compile(r"^\s*\.(decl|input|output|printsize)\s+([A-Za-z_]\w*)\s*(\(([^)]*)\))?(.*)$")


def _strip(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return "\n".join(re.split(r"%|//", ln)[0] for ln in text.splitlines())


def directives(text: str) -> Directives:
    """The Souffle directives of a program."""
    d = Directives()
    for ln in _strip(text).splitlines():
        m = _DIRECTIVE.match(ln)
        if not m:
            continue
        kind, name, args, rest = m.group(1), m.group(2), m.group(4) or "", m.group(5) or ""
        if kind == "decl":
            cols = [a.split(":")[0].strip() for a in args.split(",") if a.strip()]
            d.decl[name] = len(cols)
            cm = re.search(r"choice-domain\s*\(?\s*([^)]*)\)?", rest)
            if cm:
                dom = [c.strip() for c in cm.group(1).split(",") if c.strip()]
                if dom != cols[:len(dom)] or len(dom) != len(cols) - 1:
                    raise ValueError(f"{name}: choice-domain must be all columns but the last")
                d.dep[name] = 1
        elif kind == "input":
            fm = re.search(r'filename\s*=\s*"([^"]*)"', args)
            d.inputs[name] = fm.group(1) if fm else None
        elif kind == "output":
            d.outputs.append(name)
        else:
            d.printsize.append(name)
    return d


def parse(text: str) -> list:
    """Rules of a program ('%', '//' and '/* */' are comments, lines that
    start with '.' are directives, a rule ends with '.')."""
    lines = [ln for ln in _strip(text).splitlines() if not ln.lstrip().startswith(".")]
    rules = []
    fresh = [0]

    def anon(m):
        fresh[0] += 1
        return f"_{fresh[0]}"

    # a rule ends at a '.' that is not inside a number
    for stmt in re.split(r"\.(?!\d)", " ".join(lines)):
        stmt = stmt.strip()
        if not stmt:
            continue
        if ":-" not in stmt:
            raise ValueError(f"not a rule: {stmt!r}")
        head_s, body_s = stmt.split(":-", 1)
        body_s = re.sub(r"(?<![\w])_(?![\w])", anon, body_s)
        m = _ATOM.fullmatch(head_s)
        if not m:
            raise ValueError(f"bad head: {head_s!r}")
        head = Atom(m.group(1), tuple(g.replace(" ", "") for g in m.groups()[1:] if g))
        body, ne = [], None
        for part in re.split(r",(?![^(]*\))", body_s):
            ma, mn = _ATOM.fullmatch(part), _NE.fullmatch(part)
            if ma:
                args = tuple(g.replace(" ", "") for g in ma.groups()[1:] if g)
                if any(_term(t)[0] is None or _term(t)[1] for t in args):
                    raise ValueError(f"body atoms take variables only: {part!r}")
                body.append(Atom(ma.group(1), args))
            elif mn and ne is None:
                ne = (mn.group(1), mn.group(2))
            else:
                raise ValueError(f"bad body literal: {part!r}")
        bvars = {v for a in body for v in a.args}
        hvars = {_term(t)[0] for t in head.args} - {None}
        if not body or not hvars <= bvars:
            raise ValueError(f"head variables must appear in the body: {stmt!r}")
        if ne and set(ne) != {_term(t)[0] for t in head.args[:2]}:
            raise ValueError(f"'!=' must relate the first two head variables: {stmt!r}")
        if len(body) > 3:
            raise ValueError(f"at most three body atoms: {stmt!r}")
        if ne and len(body) == 1:
            # a Copy ignores predicates (src/copy.cu)
            raise ValueError(f"'!=' needs a join (two or three body atoms): {stmt!r}")
        rules.append(Rule(head, body, ne, stmt))
    return rules


def _components(rules: list) -> list:
    """Strongly connected components of the head predicates, dependencies
    first (Tarjan)."""
    idb = sorted({r.head.pred for r in rules})
    deps = {p: sorted({a.pred for r in rules if r.head.pred == p for a in r.body if a.pred in idb})
            for p in idb}
    index, low, stack, on, out, n = {}, {}, [], set(), [], [0]

    def visit(v):
        index[v] = low[v] = n[0]
        n[0] += 1
        stack.append(v)
        on.add(v)
        for w in deps[v]:
            if w not in index:
                visit(w)
                low[v] = min(low[v], low[w])
            elif w in on:
                low[v] = min(low[v], index[w])
        if low[v] == index[v]:
            comp = []
            while True:
                w = stack.pop()
                on.discard(w)
                comp.append(w)
                if w == v:
                    break
            out.append(sorted(comp))

    for v in idb:
        if v not in index:
            visit(v)
    return out


def _shared(a: Atom, b: Atom) -> list:
    return [v for v in a.args if v in b.args]


def _other(a: Atom, v: str) -> str:
    return a.args[1] if a.args[0] == v else a.args[0]


def _order(a: Atom, key: str) -> int:
    """How the atom's relation is stored for a join on `key`: 12 as written,
    21 swapped (key first), 123 a ternary relation keyed on its first
    column."""
    if len(a.args) == 3:
        if a.args[0] != key:
            raise ValueError(f"{a.pred}: a ternary relation joins on its first column")
        return 123
    if a.args[0] == key:
        return 12
    if a.args[1] == key:
        return 21
    raise ValueError(f"{a} does not hold {key}")


def _stored(a: Atom, order: int) -> tuple:
    """The atom's variables in the stored column order."""
    return (a.args[1], a.args[0]) if order == 21 else a.args


@dataclass
class Compiled:
    relations: dict = field(default_factory=dict)   # head predicate -> Relation (as written)
    iterations: dict = field(default_factory=dict)  # component name -> loop passes
    lies: dict = field(default_factory=dict)

    @property
    def output(self):
        return next(iter(self.relations.values()))


def _rel_name(pred: str, order: int) -> str:
    return {12: f"{pred}_2__1_2", 21: f"{pred}_2__2_1", 123: f"{pred}_3__1_2_3"}[order]


# A relation of the program is (predicate, order): order 12 as written, 21
# swapped, 123 a ternary relation; a tmp relation is (name, 12).


@dataclass
class OpSpec:
    kind: str                 # "join", "copy" or "acopy"
    src: tuple                # inner of a join, source of a copy
    src_ver: int
    outer: tuple | None       # outer of a join
    outer_ver: int | None
    out: tuple
    sel: tuple
    pred: tuple | None = None


@dataclass
class Component:
    name: str
    preds: list
    update: list = field(default_factory=list)   # relations the LIE updates
    statics: list = field(default_factory=list)  # relations it reads from outside
    tmps: list = field(default_factory=list)
    ops: list = field(default_factory=list)      # in the LIE's order


@dataclass
class Program:
    arity: dict
    deps: dict
    main: dict        # predicate -> its order as written (12 or 123)
    seed_rules: list  # number-headed rules over one input atom
    inputs: set
    comps: list       # in dependency order


def compile(text: str, input_names, deps: dict | None = None) -> Program:
    """The operator program of `text`, inputs being the predicates named."""
    rules = parse(text)
    deps = dict(deps or {})
    input_names = set(input_names)
    idb = {r.head.pred for r in rules}
    arity = {}
    for r in rules:
        for a in [r.head] + r.body:
            if arity.setdefault(a.pred, len(a.args)) != len(a.args):
                raise ValueError(f"{a.pred} is used with {arity[a.pred]} and {len(a.args)} columns")
        for a in r.body:
            if a.pred not in idb and a.pred not in input_names:
                raise ValueError(f"no rule and no input for {a.pred!r}")
    main = {p: (123 if arity[p] == 3 else 12) for p in arity}
    seed_rules = []
    for r in rules:
        if any(_term(t)[2] is not None for t in r.head.args):
            if len(r.body) != 1 or r.body[0].pred not in input_names:
                raise ValueError(f"a number in the head needs one input atom: {r.text!r}")
            seed_rules.append(r)
    rules = [r for r in rules if r not in seed_rules]

    def sel_of(t, key, inner, io, outer, oo):
        v, k, _ = _term(t)
        si, so = _stored(inner, io), _stored(outer, oo)
        base = INNER(si.index(v)) if v in si else OUTER(so.index(v)) if v in so else None
        if base is None:
            raise ValueError(f"variable {v} is not in the join")
        return PLUS(base, k) if k else base

    prog = Program(arity, deps, main, seed_rules, input_names, [])
    heads = {r.head.pred for r in rules}
    tmp_n = [0]
    # predicates defined by number-headed rules only come first (their rows
    # are all seeds)
    for comp in [[p] for p in sorted({r.head.pred for r in seed_rules}) if p not in heads] + \
            _components(rules):
        comp_set = set(comp)
        C = Component("+".join(comp), comp)
        mirrors = set()

        def need(a: Atom, key: str):
            o = _order(a, key)
            if a.pred in comp_set and o == 21:
                mirrors.add(a.pred)
            return o

        def rel(pred, order):
            r_ = (pred, order)
            if pred not in comp_set and r_ not in C.statics and not pred.startswith("tmp_"):
                C.statics.append(r_)
            return r_

        for r in [r for r in rules if r.head.pred in comp_set]:
            rec = [a.pred in comp_set for a in r.body]
            hterms = r.head.args
            pred = (PRED_NE, 0, 1) if r.ne else None
            head = (r.head.pred, main[r.head.pred])
            if len(r.body) == 1:
                a = r.body[0]
                sel = []
                for t in hterms:
                    v, k, _ = _term(t)
                    s_ = SRC(a.args.index(v))
                    sel.append(PLUS(s_, k) if k else s_)
                C.ops.append(OpSpec("copy", rel(a.pred, main[a.pred]), DELTA if rec[0] else FULL,
                                    None, None, head, tuple(sel)))
                continue
            if len(r.body) == 2:
                a, b = r.body
                sv = _shared(a, b)
                if len(sv) != 1:
                    raise ValueError(f"two atoms must share one variable: {r.text!r}")
                v = sv[0]
                for d in ([i for i in (0, 1) if rec[i]] or [None]):
                    outer, inner = (r.body[d], r.body[1 - d]) if d is not None else (b, a)
                    oo, io = need(outer, v), need(inner, v)
                    sel = tuple(sel_of(t, v, inner, io, outer, oo) for t in hterms)
                    C.ops.append(OpSpec("join", rel(inner.pred, io), FULL, rel(outer.pred, oo),
                                        DELTA if d is not None else FULL, head, sel, pred))
                continue
            a, b, c = r.body
            if any(len(x.args) != 2 for x in (a, b, c)) or len(hterms) != 2 or \
                    any(_term(t)[1] for t in hterms):
                raise ValueError(f"three-atom rules are over binary relations: {r.text!r}")
            h0, h1 = hterms
            s_ab, s_bc, s_ac = _shared(a, b), _shared(b, c), _shared(a, c)
            if len(s_ab) != 1 or len(s_bc) != 1 or s_ac or s_ab == s_bc:
                raise ValueError(f"three atoms must form a chain a-b-c: {r.text!r}")
            v1, v2 = s_ab[0], s_bc[0]
            ax, cy = _other(a, v1), _other(c, v2)
            if {h0, h1} != {ax, cy}:
                raise ValueError(f"the head must hold the chain's two ends: {r.text!r}")
            if rec[0] or rec[1] or not any(rec):
                # tmp(v2, ax) from a and b (a DELTA on a or on b), then c
                t = (f"tmp_{tmp_n[0]}", 12)
                tmp_n[0] += 1
                C.tmps.append(t)
                for d in ([i for i in (0, 1) if rec[i]] or [None]):
                    outer, inner = ((a, b) if d == 0 else (b, a)) if d is not None else (b, a)
                    oo, io = need(outer, v1), need(inner, v1)
                    tsel = tuple(sel_of(x, v1, inner, io, outer, oo) for x in (v2, ax))
                    C.ops.append(OpSpec("join", rel(inner.pred, io), FULL, rel(outer.pred, oo),
                                        DELTA if d is not None else FULL, t, tsel))
                tmp_atom = Atom(t[0], (v2, ax))
                co = need(c, v2)
                sel = tuple(sel_of(x, v2, c, co, tmp_atom, 12) for x in (h0, h1))
                C.ops.append(OpSpec("join", rel(c.pred, co), FULL, t, NEWT, head, sel, pred))
            if rec[2]:
                # a DELTA on c: tmp(v1, cy) from b and c, then a
                t = (f"tmp_{tmp_n[0]}", 12)
                tmp_n[0] += 1
                C.tmps.append(t)
                oo, io = need(c, v2), need(b, v2)
                tsel = tuple(sel_of(x, v2, b, io, c, oo) for x in (v1, cy))
                C.ops.append(OpSpec("join", rel(b.pred, io), FULL, rel(c.pred, oo), DELTA, t,
                                    tsel))
                tmp_atom = Atom(t[0], (v1, cy))
                ao = need(a, v1)
                sel = tuple(sel_of(x, v1, a, ao, tmp_atom, 12) for x in (h0, h1))
                C.ops.append(OpSpec("join", rel(a.pred, ao), FULL, t, NEWT, head, sel, pred))
        for p in sorted(mirrors):
            C.ops.append(OpSpec("acopy", (p, 12), NEWT, None, None, (p, 21), (SRC(1), SRC(0))))
        for p in comp:
            C.update.append((p, main[p]))
            if p in mirrors:
                C.update.append((p, 21))
        prog.comps.append(C)
    return prog


def seed_rows(prog: Program, inputs: dict) -> dict:
    """Rows of the number-headed rules (predicate -> rows), from the inputs."""
    seeds = {}
    for r in prog.seed_rules:
        a = r.body[0]
        src = np.asarray(inputs[a.pred], dtype=np.uint64).reshape(-1, prog.arity[a.pred])
        cols = []
        for t in r.head.args:
            v, k, c = _term(t)
            cols.append(np.full(len(src), c, np.uint64) if c is not None
                        else src[:, a.args.index(v)] + np.uint64(k))
        seeds.setdefault(r.head.pred, []).append(np.stack(cols, axis=1) if len(src) else
                                                 np.zeros((0, len(cols)), np.uint64))
    return seeds


def new_relation(eng: Engine, prog: Program, key: tuple, name: str | None = None):
    pred, order = key
    name = name or (pred if pred.startswith("tmp_") else _rel_name(pred, order))
    if order == 123:
        return eng.relation(name, arity=3, dependent_column_size=prog.deps.get(pred, 0))
    return eng.relation(name, index_flag=not pred.startswith("tmp_"))


def run(eng: Engine, text: str, inputs: dict, sync=None, deps: dict | None = None) -> Compiled:
    """Compile `text` and run it on `eng` over the input relations
    (predicate -> rows); returns the head predicates' relations.  deps:
    dependent columns of a ternary predicate (1: its last column, as
    Souffle's choice-domain over the others)."""
    prog = compile(text, inputs.keys(), deps)
    seeds = seed_rows(prog, inputs)
    rels = {}

    def rows_of(pred, order):
        if pred in inputs:
            rows = np.asarray(inputs[pred], dtype=np.uint64).reshape(-1, prog.arity[pred])
        else:
            rel = rels[(pred, prog.main[pred])]
            rows = rel.rows() if rel.size() else np.zeros((0, prog.arity[pred]), np.uint64)
        return rows[:, ::-1].copy() if order == 21 else rows

    def load(rel, rows):
        eng.load(rel, rows if len(rows) else None)

    out = Compiled()
    for C in prog.comps:
        for key in C.statics:
            if key not in rels:
                rels[key] = new_relation(eng, prog, key)
                load(rels[key], rows_of(*key))
        for p in C.preds:
            key = (p, prog.main[p])
            if key not in rels:
                rels[key] = new_relation(eng, prog, key)
                parts = ([rows_of(*key)] if p in inputs else []) + seeds.get(p, [])
                load(rels[key], np.concatenate(parts) if parts else
                     np.zeros((0, prog.arity[p]), np.uint64))
        for key in C.update:
            if key not in rels:  # a mirror: the predicate's loaded rows, swapped
                base = rels[(key[0], prog.main[key[0]])]
                rows = base.rows() if base.size() else np.zeros((0, 2), np.uint64)
                rels[key] = new_relation(eng, prog, key)
                load(rels[key], rows[:, ::-1].copy())
        for key in C.tmps:
            rels[key] = new_relation(eng, prog, key)
            load(rels[key], np.zeros((0, 2), np.uint64))
        if C.ops:
            lie = eng.lie()
            for key in C.statics:
                lie.add_relations(rels[key], True)
            for key in C.update:
                lie.add_relations(rels[key], False)
            for key in C.tmps:
                lie.add_tmp_relation(rels[key])
            for op in C.ops:
                if op.kind == "copy":
                    lie.add_copy(rels[op.src], op.src_ver, rels[op.out], op.sel)
                elif op.kind == "acopy":
                    lie.add_acopy(rels[op.src], rels[op.out], op.sel)
                else:
                    kw = {"pred": op.pred} if op.pred else {}
                    lie.add_join(rels[op.src], op.src_ver, rels[op.outer], op.outer_ver,
                                 rels[op.out], op.sel, **kw)
            out.iterations[C.name] = lie.fixpoint()
            out.lies[C.name] = lie
        for p in C.preds:
            out.relations[p] = rels[(p, prog.main[p])]
    if sync:
        sync()
    return out


def run_file(eng: Engine, path: str, facts_dir: str | None = None, out_dir: str | None = None,
             inputs: dict | None = None, sync=None) -> tuple:
    """Run a Souffle-style program file: its `.input` relations from
    `inputs`, else <facts_dir>/<name>.facts, else the file name the
    directive gives (relative to the program); `.output` relations written
    to <out_dir>/<name>.csv.  Returns (Compiled, {name: size} for the
    `.printsize` relations)."""
    import os
    text, d, given = read_program(path, facts_dir, inputs)
    res = run(eng, text, given, sync=sync, deps=d.dep)
    if out_dir:
        os.makedirs(out_dir, exist_ok=True)
        for name in d.outputs:
            res.relations[name].dump_tsv(os.path.join(out_dir, name + ".csv"))

    def size(name):
        if name in res.relations:
            return res.relations[name].size()
        return input_size(given, name)

    sizes = {name: size(name) for name in d.printsize}
    return res, sizes


def input_size(given: dict, name: str) -> int:
    """Tuples of an input relation (distinct rows; 0 when declared only)."""
    if name in given and len(given[name]):
        rows = np.asarray(given[name]).reshape(len(given[name]), -1)
        return len(np.unique(rows, axis=0))
    return 0


def read_program(path: str, facts_dir: str | None = None, inputs: dict | None = None) -> tuple:
    """A program file's text, its directives and its input rows (the
    caller's, else <facts_dir>/<name>.facts, else the directive's file)."""
    import os
    from gdlog_b200 import read_tsv
    text = open(path).read()
    d = directives(text)
    for name, arity in d.decl.items():
        if arity not in (2, 3):
            raise ValueError(f"{name}: relations of 2 or 3 columns only (arity {arity})")
    given = dict(inputs or {})
    for name, fname in d.inputs.items():
        if name in given:
            continue
        cands = []
        if facts_dir:
            cands.append(os.path.join(facts_dir, name + ".facts"))
        if fname:
            cands.append(os.path.join(os.path.dirname(os.path.abspath(path)), fname))
        found = next((c for c in cands if os.path.exists(c)), None)
        if found is None:
            raise FileNotFoundError(f"no facts for {name}: tried {cands}")
        given[name] = read_tsv(found, d.decl.get(name, 2))
    return text, d, given


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="Run a Datalog program file on the engine.")
    ap.add_argument("program")
    ap.add_argument("--facts", default=None, help="directory of <name>.facts inputs")
    ap.add_argument("--out", default=None, help="directory for <name>.csv outputs")
    ap.add_argument("--engine", default="gpu", choices=["gpu", "oracle"])
    a = ap.parse_args()
    import os
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        # one rank per GPU (torchrun): every relation partitioned over the ranks
        import torch
        import torch.distributed as dist

        import partition
        device = None
        if a.engine == "gpu":
            device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
            torch.cuda.set_device(device)
        # every pass takes collectives: a rank that failed ends the others'
        # next one with an error after this long instead of the default
        from datetime import timedelta
        dist.init_process_group("nccl" if device is not None else "gloo",
                                timeout=timedelta(seconds=300))
        try:
            rank = dist.get_rank()
            with Engine(a.engine) as eng:
                res, sizes = partition.run_file_partitioned(eng, a.program, rank, world, a.facts,
                                                            a.out, device=device)
            if rank == 0:
                print(json.dumps({"sizes": sizes, "iterations": res.iterations,
                                  "ranks": world}))
        finally:
            dist.destroy_process_group()
        return
    with Engine(a.engine) as eng:
        res, sizes = run_file(eng, a.program, a.facts, a.out, sync=getattr(eng, "sync", None))
        print(json.dumps({"sizes": sizes, "iterations": res.iterations}))


if __name__ == "__main__":
    main()
