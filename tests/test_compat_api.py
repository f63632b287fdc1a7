"""The drop-in C++ API (include/gdlog/): programs written the way the
reference's drivers are written (device hooks fetched with
cudaMemcpyFromSymbol, Relation / load_relation / LIE / RelationalJoin /
RelationalCopy / RelationalACopy) give the golden answers."""
import json
import os
import subprocess

import pytest

import workloads as W
from test_oracle import GOLDEN, build_workload

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVERS = os.path.join(REPO, "gdlog-multinode_b200", "lib", "compat_drivers")


def test_compat_drivers_built():
    assert os.path.exists(DRIVERS), "run __graft_entry__.build()"


def test_headers_compile_standalone(tmp_path):
    """Every drop-in header compiles on its own (nvcc, no device needed)."""
    inc = os.path.join(REPO, "include")
    for h in ("tuple.cuh", "relation.cuh", "relational_algebra.cuh", "lie.cuh", "exception.cuh",
              "timer.cuh", "print.cuh"):
        src = tmp_path / f"t_{h}.cu"
        src.write_text(f'#include "gdlog/{h}"\nint main() {{ return 0; }}\n')
        r = subprocess.run(["nvcc", "-std=c++17", "-rdc=true", "-I", inc, "-c", str(src), "-o",
                            str(tmp_path / "t.o")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]


REF_TEST = "/root/reference/test"


@pytest.mark.skipif(not os.path.isdir(REF_TEST), reason="reference sources not present")
@pytest.mark.parametrize("driver", ["tc", "sg", "cspa", "path_length"])
def test_reference_drivers_build_unchanged(tmp_path, driver):
    """The reference's own drivers (test/tc.cu, sg.cu, cspa.cu), unchanged
    except that their `../include/*.cuh` lines name this repository's
    drop-in headers, compile and link against the engine's library (nvcc,
    no device needed; a copy in a temporary directory, nothing kept)."""
    import re
    src = open(os.path.join(REF_TEST, f"{driver}.cu")).read()
    src = re.sub(r'"\.\./include/([a-z_]+\.cuh)"', r'"gdlog/\1"', src)
    f = tmp_path / f"{driver}.cu"
    f.write_text(src)
    lib = os.path.join(REPO, "gdlog-multinode_b200", "lib")
    r = subprocess.run(["nvcc", "-std=c++17", "-rdc=true", "-gencode",
                        "arch=compute_100a,code=sm_100a", "-I", os.path.join(REPO, "include"),
                        "-o", str(tmp_path / driver), str(f), "-L", lib, "-lgdlog_b200"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert (tmp_path / driver).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tc_grid_16x16", "tc_dag_L12_W10_s2", "sg_rmat_s8_600_s1",
                                  "cspa_v120_s1"])
def test_compat_drivers_match_golden(tmp_path, name):
    prog, args = build_workload(name)
    files = []
    for i, rows in enumerate(args):
        p = tmp_path / f"in{i}.tsv"
        W.write_tsv(str(p), rows)
        files.append(str(p))
    r = subprocess.run([DRIVERS, prog.__name__, *files], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT ")][-1]
    got = json.loads(line[len("RESULT "):])
    want = GOLDEN["workloads"][name]
    assert got["sizes"] == want["sizes"]
    assert got["iterations"] == want["iterations"]
    assert got["digests"] == want["digests"]


@pytest.mark.gpu
def test_compat_path_length_matches_oracle(tmp_path):
    """The arity-3 program through the drop-in API: a __device__ hook that
    adds 1 to a column, fetched with cudaMemcpyFromSymbol, recognised as
    GDL_PLUS; same sizes, digest and passes as the oracle."""
    import programs as P
    from gdlog_b200 import Engine
    e = W.rmat_edges(8, 600, seed=3)
    p = tmp_path / "e.tsv"
    W.write_tsv(str(p), e)
    r = subprocess.run([DRIVERS, "path_length", str(p)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("RESULT ")][-1][7:])
    with Engine("oracle", max_arity=3) as o:
        ro = P.path_length(o, e)
        want = (ro.relations["path"].size(), hex(ro.relations["path"].digest()),
                ro.iterations["plen"])
    assert (got["sizes"]["path"], got["digests"]["path"], got["iterations"]["plen"]) == want
