"""Input and output files (gdl_read_tsv, gdl_relation_load_tsv,
gdl_relation_dump_tsv): the reference drivers' reading rules
(test/tc.cu:17-57) restated in Python below and compared on edge cases and
on the reference's own data files when they are present; loads from files
and sorted dumps checked on the GPU against the oracle."""
import os

import numpy as np
import pytest

import programs as P
import workloads as W
from gdlog_b200 import Engine, GdlError, read_tsv, write_tsv

from conftest import REF_ROOT

REF_DATA = os.path.join(REF_ROOT, "data")


def reference_rules(text: str, arity: int):
    """get_row_size + get_relation_from_file as the drivers use them: rows =
    count of newlines; each value "%lld" after white space; one character
    consumed after every column but the last; values stored as u64."""
    rows = text.count("\n")
    i, n = 0, len(text)
    vals = []
    for r in range(rows):
        for c in range(arity):
            while i < n and text[i] in " \t\n\r\v\f":
                i += 1
            j = i
            if j < n and text[j] in "+-":
                j += 1
            k = j
            while k < n and text[k].isdigit():
                k += 1
            if k == j:
                raise ValueError("no value")
            v = int(text[i:k]) % (1 << 64)
            vals.append(v)
            i = k
            if c != arity - 1 and i < n:
                i += 1
    return np.array(vals, dtype=np.uint64).reshape(rows, arity) if rows else \
        np.zeros((0, arity), dtype=np.uint64)


@pytest.mark.parametrize("text", [
    "1\t2\n3\t4\n",
    "1\t2\n3\t4",            # last line without a newline is not read
    "  5\t 6\n 7\t8\n",       # white space before a value
    "9 10\r\n11 12\r\n",     # any one-character separator, CRLF lines
    "-1\t3\n4\t-2\n",        # negative values wrap to u64
    "",
])
def test_read_tsv_follows_the_reference_rules(tmp_path, text):
    f = tmp_path / "r.txt"
    f.write_text(text)
    got = read_tsv(str(f), 2)
    want = reference_rules(text, 2)
    assert got.shape == want.shape and (got == want).all()


def test_read_tsv_reports_missing_values(tmp_path):
    f = tmp_path / "bad.txt"
    f.write_text("1\t2\n3\n\n")  # three newlines, the third row has no values
    with pytest.raises(GdlError):
        read_tsv(str(f), 2)
    with pytest.raises(GdlError):
        read_tsv(str(tmp_path / "absent.txt"), 2)


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data not present")
@pytest.mark.parametrize("name", ["data_5.txt", "data_7035.txt", "data_21693.txt"])
def test_read_tsv_on_reference_data(name):
    path = os.path.join(REF_DATA, name)
    got = read_tsv(path, 2)
    want = reference_rules(open(path).read(), 2)
    assert got.shape == want.shape and (got == want).all()


def test_write_tsv_layout(tmp_path):
    f = tmp_path / "o.tsv"
    write_tsv(str(f), np.array([[1, 2], [3, 40]], dtype=np.uint64))
    assert f.read_text() == "1\t2\n3\t40\n"


@pytest.mark.gpu
def test_load_from_file_and_dump_sorted(tmp_path):
    """A file with duplicates, out of order, loads as the sorted unique
    relation; SG from that file dumps exactly what the oracle computes."""
    e = W.rmat_edges(8, 600, seed=4)
    rows = np.concatenate([e[::-1], e[:50]])  # reversed order plus duplicates
    f = tmp_path / "edges.txt"
    write_tsv(str(f), rows)
    with Engine("gpu") as g:
        rel = g.relation("edge_2__1_2")
        g.load_tsv(rel, str(f))
        assert (rel.rows() == np.unique(rows, axis=0)).all()
        r = P.sg(g, read_tsv(str(f)), sync=g.sync)
        n = r.output.dump_tsv(str(tmp_path / "sg.tsv"))
    with Engine("oracle") as o:
        ro = P.sg(o, read_tsv(str(f)))
        o.dump_tsv(ro.output, str(tmp_path / "sg_oracle.tsv"))
        n_oracle = ro.output.size()
    assert n == n_oracle
    assert (tmp_path / "sg.tsv").read_text() == (tmp_path / "sg_oracle.tsv").read_text()
