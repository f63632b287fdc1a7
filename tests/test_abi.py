"""The C-ABI library loads and exports every entry point include/*.h
declares; without a CUDA device the engine refuses to start with a status
code instead of falling back to anything.  No compute calls here."""
import ctypes as C
import os
import re
import subprocess

import pytest

import gdlog_b200 as G

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(REPO, "include", f) for f in sorted(os.listdir(os.path.join(REPO, "include")))
           if f.endswith(".h")]


def declared(prefix="gdl_", headers=None):
    names = set()
    for h in headers or HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(" + prefix + r"\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_headers_declare_entry_points():
    names = declared()
    assert "gdl_lie_fixpoint" in names and "gdl_relation_load" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    assert os.path.exists(G.GPU_LIB), "engine library not built"
    missing = declared() - exported(G.GPU_LIB)
    assert not missing, f"not exported: {sorted(missing)}"


def test_library_loads_and_binds():
    lib = G.load_library("gpu")
    assert lib.gdl_version().startswith(b"gdlog-b200")
    assert lib.gdl_status_string is not None
    for name in declared():
        assert hasattr(lib, name)


def test_oracle_mirrors_the_abi():
    orc = declared("orc_", [os.path.join(REPO, "oracle", "oracle.h")])
    gdl = {n[4:] for n in declared()}
    # every program-building entry point has an oracle twin
    for n in ("relation_create", "relation_load", "relation_size", "relation_export",
              "relation_digest", "lie_create", "lie_add_relation", "lie_add_tmp_relation",
              "lie_add_join", "lie_add_copy", "lie_add_acopy", "lie_set_max_iteration",
              "lie_set_reload_full", "lie_fixpoint", "lie_trace"):
        assert n in gdl and "orc_" + n in orc


def test_no_device_means_error_not_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(G.GdlError):
        G.Engine("gpu")


def test_null_arguments_rejected():
    lib = G.load_library("gpu")
    assert lib.gdl_engine_create(0, None, None) == 1  # GDL_E_INVALID
    assert lib.gdl_relation_size(None, 0, 1, None) == 1
    assert lib.gdl_lie_fixpoint(None, 0, None) == 1
    msg = lib.gdl_last_error(None)
    assert msg


def test_tuning_struct_matches_the_header(tmp_path):
    """gdl_tuning as the C compiler lays it out (include/gdlog_b200.h) and
    the ctypes mirror the binding passes to gdl_engine_set_tuning agree
    field by field."""
    fields = [f for f, _ in G.Tuning._fields_]
    src = tmp_path / "t.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"gdlog_b200.h\"\n"
                   "int main(void) {\n  printf(\"%zu\\n\", sizeof(gdl_tuning));\n"
                   + "".join(f"  printf(\"%zu\\n\", offsetof(gdl_tuning, {f}));\n" for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "t"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(REPO, "include"), str(src), "-o",
                    str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                           check=True).stdout.split()]
    assert vals[0] == C.sizeof(G.Tuning)
    assert vals[1:] == [getattr(G.Tuning, f).offset for f in fields]
