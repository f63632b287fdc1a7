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


from conftest import DROPIN, REF_ROOT

REF_TEST = os.path.join(REF_ROOT, "test")


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


# -- the reference's own drivers, unchanged, running on the GPU -------------

def run_dropin(driver, *args, timeout=600):
    exe = os.path.join(DROPIN, "bin", driver)
    if not os.path.exists(exe):
        pytest.skip("reference drivers not built (make -C oracle dropin REF=<reference root>)")
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def last_lie_passes(out: str) -> int:
    """Loop passes of the last LIE from the per-iteration log lines
    ("Iteration i finish populating", src/lie.cu:199-200)."""
    its = [int(ln.split()[1]) for ln in out.splitlines()
           if ln.startswith("Iteration ") and ln.endswith("finish populating")]
    last0 = max(i for i, v in enumerate(its) if v == 0)
    return max(its[last0:]) + 1


def count_after(out: str, label: str) -> int:
    line = [ln for ln in out.splitlines() if ln.startswith(label)][-1]
    return int(line[len(label):].split()[0])


# Same generation on the reference's data files gives the sizes and loop
# passes the reference publishes (README.md:101-103, test/cuDF/sg.json);
# the closure gives what the bit-matrix oracle gives on the same file.
DROPIN_CASES = [
    ("sg", "data_21693.txt", "sg counts ", 23519, 58),
    ("sg", "data_7035.txt", "sg counts ", 285431, 56),
    ("sg", "data_5.txt", "sg counts ", 4, 3),
    ("tc", "data_7035.txt", "Path counts ", None, None),
    ("tc", "data_21693.txt", "Path counts ", None, None),
]


@pytest.mark.gpu
@pytest.mark.parametrize("driver,data,label,size,passes", DROPIN_CASES)
def test_reference_drivers_run_on_reference_data(driver, data, label, size, passes):
    """test/tc.cu and test/sg.cu, compiled unchanged against the drop-in
    headers (oracle/Makefile `dropin`), run on the B200 on the reference's
    own data files."""
    import programs as P
    from gdlog_b200 import Engine, read_tsv
    path = os.path.join(DROPIN, "data", data)
    out = run_dropin(driver, path)
    got = (count_after(out, label), last_lie_passes(out))
    if size is None:
        with Engine("oracle_bitset") as o:
            r = getattr(P, driver)(o, read_tsv(path))
            size, passes = r.output.size(), list(r.iterations.values())[-1]
    assert got == (size, passes)


@pytest.mark.gpu
def test_reference_cspa_driver_runs(tmp_path):
    """test/cspa.cu, unchanged, on a facts directory (assign.facts,
    dereference.facts): its relations' sizes as the oracle has them."""
    import programs as P
    from gdlog_b200 import Engine
    assign, deref = W.cspa_facts(300, 600, 225, seed=3)
    W.write_tsv(str(tmp_path / "assign.facts"), assign)
    W.write_tsv(str(tmp_path / "dereference.facts"), deref)
    out = run_dropin("cspa", str(tmp_path))
    with Engine("oracle_bitset") as o:
        r = P.cspa(o, assign, deref)
        want = {k: v.size() for k, v in r.relations.items()}
    full = {}
    for ln in out.splitlines():
        if ln.startswith("iteration ") and " full counts " in ln:
            name = ln.split()[3]
            full[name] = int(ln.rsplit(" ", 1)[1])
    assert full["value_flow_2__1_2"] == want["value_flow"]
    assert full["memory_alias_2__1_2"] == want["memory_alias"]
    assert full["value_alias_2__1_2"] == want["value_alias"]
    assert last_lie_passes(out) == r.iterations["analysis"]


@pytest.mark.gpu
def test_reference_path_length_driver_runs():
    """test/path_length.cu, unchanged (arity 3, a dependent column and a
    hook that adds 1): its closure size as the oracle has it."""
    import programs as P
    from gdlog_b200 import Engine, read_tsv
    path = os.path.join(DROPIN, "data", "data_7035.txt")
    out = run_dropin("path_length", path)
    with Engine("oracle", max_arity=3) as o:
        r = P.path_length(o, read_tsv(path))
        want = r.output.size()
    full = [int(ln.rsplit(" ", 1)[1]) for ln in out.splitlines()
            if ln.startswith("iteration ") and " full counts " in ln]
    assert full[-1] == want
    assert last_lie_passes(out) == r.iterations["plen"]
