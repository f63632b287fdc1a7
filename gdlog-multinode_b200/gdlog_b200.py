"""ctypes binding of the engine's C-ABI (include/gdlog_b200.h).

Mirrors the reference's operator API for the semi-naive path, so that a
program reads like the reference drivers (test/tc.cu, test/sg.cu,
test/cspa.cu):

    eng = Engine("gpu")
    path = eng.relation("path_2__1_2", index_flag=False)
    eng.load(path, edges)                         # load_relation
    lie = eng.lie()                               # LIE(grid, block)
    lie.add_relations(edge, static=True)          # LIE::add_relations
    lie.add_join(edge, FULL, path, DELTA, path,   # RelationalJoin(...)
                 gen=(INNER(1), OUTER(1)))
    iterations = lie.fixpoint()                   # LIE::fixpoint_loop

The same class drives the CPU oracles (``Engine("oracle")`` over sorted
tuple lists and ``Engine("oracle_bitset")`` over bit matrices, both test
infrastructure) through their mirror C-ABIs, so tests run one program on
all of them.
The GPU backend fails loudly when its shared library is missing: there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GPU_LIB = os.path.join(HERE, "lib", "libgdlog_b200.so")
ORACLE_LIB = os.path.join(REPO, "oracle", "liboracle.so")

DELTA, FULL, NEWT = 0, 1, 2
PRED_NONE, PRED_NE, PRED_EQ, PRED_LT, PRED_LE, PRED_GT, PRED_GE = range(7)
STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "UNSUPPORTED",
          5: "TIMEOUT", 6: "CAPACITY"}


def INNER(c: int) -> int:
    return c


def OUTER(c: int) -> int:
    return 16 + c


def SRC(c: int) -> int:
    return c


def PLUS(sel: int, k: int) -> int:
    """GDL_PLUS: a hook column plus a constant, e.g. PLUS(OUTER(2), 1)."""
    return sel | (k << 8)


class Tuning(C.Structure):
    """gdl_tuning (include/gdlog_b200.h); a zero field keeps the default."""
    _fields_ = [("dedup", C.c_int32), ("dense_max_bits", C.c_int32),
                ("join_ctas_per_sm", C.c_int32), ("count_ctas_per_sm", C.c_int32),
                ("index_slots_per_key", C.c_int32), ("dirty_min_log2_words", C.c_int32),
                ("dense_join_passes", C.c_int32), ("join_aggregate", C.c_int32),
                ("pull_joins", C.c_int32), ("row_gather", C.c_int32),
                ("spin_limit_log2", C.c_int32), ("radix_bits", C.c_int32),
                ("join_block", C.c_int32), ("rows_piece", C.c_int32),
                ("load_dedup", C.c_int32)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class GdlError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_P = C.c_void_p
_I = C.c_int32
_U64 = C.c_uint64
_PU64 = C.POINTER(C.c_uint64)
_PI = C.POINTER(C.c_int32)

# (name, argtypes) shared by both prefixes; engine pointer first.
_SIGS = {
    "relation_create": [_P, C.c_char_p, _I, _I, _I, _I, _I, _PI],
    "relation_load": [_P, _I, _PU64, _U64],
    "relation_size": [_P, _I, _I, _PU64],
    "relation_export": [_P, _I, _I, _PU64, _U64, _PU64],
    "relation_digest": [_P, _I, _I, _PU64],
    "lie_create": [_P, _PI],
    "lie_add_relation": [_P, _I, _I, _I],
    "lie_add_tmp_relation": [_P, _I, _I],
    "lie_add_join": [_P, _I, _I, _I, _I, _I, _I, _PI, _I, _I, _I, _I],
    "lie_add_copy": [_P, _I, _I, _I, _I, _PI, _I],
    "lie_add_acopy": [_P, _I, _I, _I, _PI, _I],
    "lie_set_max_iteration": [_P, _I, C.c_int64],
    "lie_set_reload_full": [_P, _I, _I],
    "lie_fixpoint": [_P, _I, _PU64],
    "lie_trace": [_P, _I, _PU64, _U64, _PU64],
}

_libs: dict = {}


_PREFIX = {"gpu": "gdl_", "oracle": "orc_", "oracle_bitset": "orb_"}


def load_library(kind: str) -> C.CDLL:
    """Open the GPU engine ("gpu") or a CPU oracle ("oracle",
    "oracle_bitset") library."""
    if kind in _libs:
        return _libs[kind]
    path = GPU_LIB if kind == "gpu" else ORACLE_LIB
    if not os.path.exists(path):
        raise GdlError(4, f"{kind} library not built: {path} (run __graft_entry__.build())")
    lib = C.CDLL(path)
    pre = _PREFIX[kind]
    for name, args in _SIGS.items():
        f = getattr(lib, pre + name)
        f.argtypes = args
        f.restype = _I
    if kind == "gpu":
        lib.gdl_engine_create.argtypes = [_I, _P, C.POINTER(_P)]
        lib.gdl_engine_create.restype = _I
        lib.gdl_engine_destroy.argtypes = [_P]
        lib.gdl_engine_destroy.restype = _I
        lib.gdl_last_error.argtypes = [_P]
        lib.gdl_last_error.restype = C.c_char_p
        lib.gdl_version.restype = C.c_char_p
        lib.gdl_lie_stats.argtypes = [_P, _I, C.POINTER(C.c_double), _I]
        lib.gdl_lie_stats.restype = _I
        lib.gdl_lie_set_trace.argtypes = [_P, _I, _I]
        lib.gdl_lie_set_trace.restype = _I
        lib.gdl_engine_sync.argtypes = [_P]
        lib.gdl_engine_sync.restype = _I
        lib.gdl_relation_load_device.argtypes = [_P, _I, _P, _U64]
        lib.gdl_relation_load_device.restype = _I
        lib.gdl_engine_set_instances.argtypes = [_P, C.POINTER(C.c_uint32), _I]
        lib.gdl_engine_set_instances.restype = _I
        lib.gdl_engine_instance_shift.argtypes = [_P, _PI]
        lib.gdl_engine_instance_shift.restype = _I
        lib.gdl_lie_instance_iterations.argtypes = [_P, _I, _PU64, _I]
        lib.gdl_lie_instance_iterations.restype = _I
        lib.gdl_relation_instance_stats.argtypes = [_P, _I, _PU64, _PU64, _I]
        lib.gdl_relation_instance_stats.restype = _I
        lib.gdl_engine_set_tuning.argtypes = [_P, C.POINTER(Tuning)]
        lib.gdl_engine_set_tuning.restype = _I
        lib.gdl_engine_get_tuning.argtypes = [_P, C.POINTER(Tuning)]
        lib.gdl_engine_get_tuning.restype = _I
        lib.gdl_engine_set_dedup.argtypes = [_P, _I, _I]
        lib.gdl_engine_set_dedup.restype = _I
        lib.gdl_engine_clear.argtypes = [_P]
        lib.gdl_engine_clear.restype = _I
        lib.gdl_engine_test_timeout.argtypes = [_P, _I]
        lib.gdl_engine_test_timeout.restype = _I
        lib.gdl_profile_kinds.argtypes = []
        lib.gdl_profile_kinds.restype = _I
        lib.gdl_profile_kind_name.argtypes = [_I]
        lib.gdl_profile_kind_name.restype = C.c_char_p
        lib.gdl_engine_set_profile.argtypes = [_P, _I]
        lib.gdl_engine_set_profile.restype = _I
        lib.gdl_engine_profile.argtypes = [_P, C.POINTER(C.c_double), _I]
        lib.gdl_engine_profile.restype = _I
        lib.gdl_engine_profile_reset.argtypes = [_P]
        lib.gdl_engine_profile_reset.restype = _I
        lib.gdl_read_tsv.argtypes = [C.c_char_p, _I, _PU64, _U64, _PU64]
        lib.gdl_read_tsv.restype = _I
        lib.gdl_relation_load_tsv.argtypes = [_P, _I, C.c_char_p]
        lib.gdl_relation_load_tsv.restype = _I
        lib.gdl_relation_dump_tsv.argtypes = [_P, _I, _I, C.c_char_p, _PU64]
        lib.gdl_relation_dump_tsv.restype = _I
        lib.gdl_join_count.argtypes = [_P, _I, _I, _I, _I, _PU64]
        lib.gdl_join_count.restype = _I
        lib.gdl_relation_export_device.argtypes = [_P, _I, _I, _P, _U64, _PU64]
        lib.gdl_relation_export_device.restype = _I
        lib.gdl_partition_rows.argtypes = [_P, _P, _U64, _I, _I, _P, _PU64]
        lib.gdl_partition_rows.restype = _I
    else:
        f = lambda n: getattr(lib, pre + n)  # noqa: E731
        f("engine_create").argtypes = [_I, _I, C.POINTER(_P)]
        f("engine_create").restype = _I
        f("engine_destroy").argtypes = [_P]
        f("engine_destroy").restype = _I
        f("last_error").argtypes = [_P]
        f("last_error").restype = C.c_char_p
        f("engine_clear").argtypes = [_P]
        f("engine_clear").restype = _I
        f("threads").argtypes = [_P]
        f("threads").restype = _I
        f("lie_seconds").argtypes = [_P, _I, C.POINTER(C.c_double)]
        f("lie_seconds").restype = _I
        if kind == "oracle":
            f("join_count").argtypes = [_P, _I, _I, _I, _I, _PU64]
            f("join_count").restype = _I
    _libs[kind] = lib
    return lib


def read_tsv(path: str, arity: int = 2) -> np.ndarray:
    """The reference drivers' file read (test/tc.cu:17-57) through
    gdl_read_tsv: rows = number of newlines, "%lld" values, one separator
    character after every column but the last.  Needs no GPU."""
    lib = load_library("gpu")
    n = C.c_uint64(0)
    code = lib.gdl_read_tsv(path.encode(), arity, None, 0, C.byref(n))
    if code not in (0, 6):  # GDL_OK, GDL_E_CAPACITY (sizing call)
        raise GdlError(code, lib.gdl_last_error(None).decode())
    out = np.zeros((max(int(n.value), 1), arity), dtype=np.uint64)
    code = lib.gdl_read_tsv(path.encode(), arity, out.ctypes.data_as(_PU64), n.value, C.byref(n))
    if code:
        raise GdlError(code, lib.gdl_last_error(None).decode())
    return out[: int(n.value)]


def write_tsv(path: str, rows: np.ndarray) -> None:
    """Sorted-relation dump layout of gdl_relation_dump_tsv: decimal
    columns separated by a tab, one row per line."""
    with open(path, "w") as f:
        for r in np.asarray(rows, dtype=np.uint64).tolist():
            f.write("\t".join(str(c) for c in r) + "\n")


class DeviceRows:
    """Rows already in device memory: a contiguous (n, 2) tensor of 64-bit
    integers (any object with data_ptr() and shape, e.g. a torch tensor).
    Keeps the tensor alive; `reversed()` gives the column-swapped twin."""

    def __init__(self, tensor, reversed_tensor=None):
        if tensor.dim() != 2 or tensor.shape[1] != 2 or tensor.element_size() != 8:
            raise ValueError("DeviceRows needs an (n, 2) tensor of 64-bit integers")
        self.t = tensor.contiguous()
        self._rev = reversed_tensor

    @property
    def ptr(self) -> int:
        return self.t.data_ptr()

    @property
    def n(self) -> int:
        return int(self.t.shape[0])

    @property
    def nbytes(self) -> int:
        return self.n * 16

    def reversed(self) -> "DeviceRows":
        if self._rev is None:
            self._rev = DeviceRows(self.t.flip(1).contiguous(), self.t)
        elif not isinstance(self._rev, DeviceRows):
            self._rev = DeviceRows(self._rev, self.t)
        return self._rev


class Relation:
    """Handle of a declared relation (include/relation.cuh:257-300)."""

    def __init__(self, eng: "Engine", rid: int, name: str, arity: int):
        self.eng, self.id, self.name, self.arity = eng, rid, name, arity

    def size(self, version: int = FULL) -> int:
        return self.eng.size(self, version)

    def rows(self, version: int = FULL) -> np.ndarray:
        return self.eng.export(self, version)

    def digest(self, version: int = FULL) -> int:
        return self.eng.digest(self, version)

    def dump_tsv(self, path: str, version: int = FULL) -> int:
        """Write this version's sorted tuples as TSV; returns the rows."""
        return self.eng.dump_tsv(self, path, version)

    def instance_stats(self, n: int):
        """Batched form: per-instance (sizes, digests) of FULL, local ids."""
        sizes = np.zeros(n, dtype=np.uint64)
        digests = np.zeros(n, dtype=np.uint64)
        self.eng._check(self.eng.lib.gdl_relation_instance_stats(
            self.eng.h, self.id, sizes.ctypes.data_as(_PU64), digests.ctypes.data_as(_PU64), n))
        return sizes, digests

    def __repr__(self):
        return f"Relation({self.name!r}, id={self.id})"


class Lie:
    """LIE (include/lie.cuh:11-65)."""

    def __init__(self, eng: "Engine", lid: int):
        self.eng, self.id = eng, lid
        self.iterations = None

    def _call(self, name, *args):
        return self.eng._call(name, *args)

    def add_relations(self, rel: Relation, static: bool) -> None:
        self._call("lie_add_relation", self.id, rel.id, int(bool(static)))

    def add_tmp_relation(self, rel: Relation) -> None:
        self._call("lie_add_tmp_relation", self.id, rel.id)

    def add_join(self, inner: Relation, inner_ver: int, outer: Relation, outer_ver: int,
                 output: Relation, gen, pred=None) -> None:
        g = (C.c_int32 * len(gen))(*gen)
        kind, a, b = pred if pred else (PRED_NONE, 0, 0)
        self._call("lie_add_join", self.id, inner.id, inner_ver, outer.id, outer_ver,
                   output.id, g, len(gen), kind, a, b)

    def add_copy(self, src: Relation, src_ver: int, dest: Relation, gen) -> None:
        g = (C.c_int32 * len(gen))(*gen)
        self._call("lie_add_copy", self.id, src.id, src_ver, dest.id, g, len(gen))

    def add_acopy(self, src: Relation, dest: Relation, gen) -> None:
        g = (C.c_int32 * len(gen))(*gen)
        self._call("lie_add_acopy", self.id, src.id, dest.id, g, len(gen))

    @property
    def max_iteration(self):
        return None

    @max_iteration.setter
    def max_iteration(self, m: int) -> None:
        self._call("lie_set_max_iteration", self.id, int(m))

    def set_reload_full(self, flag: bool) -> None:
        self._call("lie_set_reload_full", self.id, int(bool(flag)))

    reload_full_flag = property(None, set_reload_full)

    def set_trace(self, flag: bool) -> None:
        if self.eng.kind == "gpu":
            self.eng._check(self.eng.lib.gdl_lie_set_trace(self.eng.h, self.id, int(bool(flag))))

    def fixpoint(self) -> int:
        out = C.c_uint64(0)
        self._call("lie_fixpoint", self.id, C.byref(out))
        self.iterations = int(out.value)
        return self.iterations

    def instance_iterations(self, n: int) -> np.ndarray:
        """Batched form: loop passes each instance would have taken alone."""
        out = np.zeros(n, dtype=np.uint64)
        self.eng._check(self.eng.lib.gdl_lie_instance_iterations(
            self.eng.h, self.id, out.ctypes.data_as(_PU64), n))
        return out

    def trace(self) -> np.ndarray:
        n = C.c_uint64(0)
        self._call("lie_trace", self.id, None, 0, C.byref(n))
        buf = np.zeros(int(n.value) * 5, dtype=np.uint64)
        self._call("lie_trace", self.id, buf.ctypes.data_as(_PU64), n.value, C.byref(n))
        return buf.reshape(-1, 5)

    def stats(self) -> dict:
        if self.eng.kind != "gpu":
            s = C.c_double(0)
            self.eng._check(getattr(self.eng.lib, self.eng.pre + "lie_seconds")(
                self.eng.h, self.id, C.byref(s)))
            return {"ms": s.value * 1e3}
        out = (C.c_double * 9)()
        self.eng._check(self.eng.lib.gdl_lie_stats(self.eng.h, self.id, out, 9))
        return {"ms": out[0], "kernels": int(out[1]), "iterations": int(out[2]),
                "retries": int(out[3]), "graph_launches": int(out[4]), "setup_ms": out[5],
                "grow_ms": out[6], "graph_ms": out[7], "graph_reused": int(out[8])}


class Engine:
    """One engine (GPU: one CUDA stream on one device; oracle: CPU threads)."""

    DEDUP = {"auto": 0, "sort": 1, "dense": 2}

    def __init__(self, kind: str = "gpu", device: int = 0, threads: int = 0,
                 max_arity: int = 2, stream: int | None = None, dedup: str | None = None):
        if kind not in _PREFIX:
            raise ValueError(kind)
        self.kind = kind
        self.lib = load_library(kind)
        self.pre = _PREFIX[kind]
        h = _P()
        if kind == "gpu":
            code = self.lib.gdl_engine_create(device, stream, C.byref(h))
            if code:
                raise GdlError(code, "gdl_engine_create failed (no CUDA device?)")
        else:
            code = getattr(self.lib, self.pre + "engine_create")(max_arity, threads, C.byref(h))
            if code:
                raise GdlError(code, f"{self.pre}engine_create failed")
        self.h = h
        self.relations: list[Relation] = []
        if kind == "gpu" and dedup is not None:
            if dedup == "dense_dirty":  # bitmaps, with dirty maps at every size
                self.set_tuning(dedup="dense", dirty_min_log2_words=11)
            elif dedup == "dense_push":  # bitmaps, every join in the push form
                self.set_tuning(dedup="dense", pull_joins=1)
            elif dedup == "dense_pull":  # bitmaps, pull form wherever it applies
                self.set_tuning(dedup="dense", pull_joins=3, row_gather=1)
            elif dedup == "dense_rows":  # bitmaps, row-gather form wherever it applies
                self.set_tuning(dedup="dense", pull_joins=3, row_gather=3)
            elif dedup == "dense_2pass":  # bitmaps, push joins as count + materialise passes
                self.set_tuning(dedup="dense", dense_join_passes=2, pull_joins=1)
            elif dedup == "dense_agg":  # bitmaps, push joins with warp-aggregated bit-sets
                self.set_tuning(dedup="dense", join_aggregate=2, pull_joins=1)
            else:
                self._check(self.lib.gdl_engine_set_dedup(self.h, self.DEDUP[dedup], 0))

    def close(self) -> None:
        if self.h:
            getattr(self.lib, self.pre + "engine_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def threads(self) -> int:
        return 0 if self.kind == "gpu" else int(getattr(self.lib, self.pre + "threads")(self.h))

    def last_error(self) -> str:
        msg = getattr(self.lib, self.pre + "last_error")(self.h)
        return msg.decode() if msg else ""

    def _check(self, code: int) -> None:
        if code:
            raise GdlError(code, self.last_error())

    def _call(self, name, *args):
        self._check(getattr(self.lib, self.pre + name)(self.h, *args))

    # -- relations ---------------------------------------------------------
    def relation(self, name: str, arity: int = 2, index_column_size: int = 1,
                 dependent_column_size: int = 0, index_flag: bool = True,
                 tmp_flag: bool = False) -> Relation:
        rid = C.c_int32(-1)
        self._call("relation_create", name.encode(), arity, index_column_size,
                   dependent_column_size, int(index_flag), int(tmp_flag), C.byref(rid))
        r = Relation(self, rid.value, name, arity)
        self.relations.append(r)
        return r

    def load(self, rel: Relation, rows) -> None:
        """load_relation: rows is an (n, arity) array of non-negative ints,
        or DeviceRows already in this engine's device memory."""
        if isinstance(rows, DeviceRows):
            self.load_device(rel, rows.ptr, rows.n)
            return
        if rows is None:
            self._call("relation_load", rel.id, None, 0)
            return
        a = np.ascontiguousarray(np.asarray(rows), dtype=np.uint64)
        if a.size == 0:
            self._call("relation_load", rel.id, None, 0)
            return
        if a.ndim != 2 or a.shape[1] != rel.arity:
            raise ValueError(f"rows must be (n, {rel.arity})")
        self._call("relation_load", rel.id, a.ctypes.data_as(_PU64), a.shape[0])

    def load_tsv(self, rel: Relation, path: str) -> None:
        """load_relation from a file read as the reference's drivers read it."""
        if self.kind == "gpu":
            self._check(self.lib.gdl_relation_load_tsv(self.h, rel.id, path.encode()))
        else:
            self.load(rel, read_tsv(path, rel.arity))

    def dump_tsv(self, rel: Relation, path: str, version: int = FULL) -> int:
        if self.kind == "gpu":
            out = C.c_uint64(0)
            self._check(self.lib.gdl_relation_dump_tsv(self.h, rel.id, version, path.encode(),
                                                       C.byref(out)))
            return int(out.value)
        rows = self.export(rel, version)
        write_tsv(path, rows)
        return len(rows)

    def size(self, rel: Relation, version: int = FULL) -> int:
        out = C.c_uint64(0)
        self._call("relation_size", rel.id, version, C.byref(out))
        return int(out.value)

    def export(self, rel: Relation, version: int = FULL) -> np.ndarray:
        n = self.size(rel, version)
        buf = np.zeros((max(n, 1), rel.arity), dtype=np.uint64)
        out = C.c_uint64(0)
        self._call("relation_export", rel.id, version, buf.ctypes.data_as(_PU64), n,
                   C.byref(out))
        return buf[: int(out.value)]

    def digest(self, rel: Relation, version: int = FULL) -> int:
        out = C.c_uint64(0)
        self._call("relation_digest", rel.id, version, C.byref(out))
        return int(out.value)

    def join_count(self, inner: Relation, inner_version: int, outer: Relation,
                   outer_version: int) -> int:
        """Output size of a join before deduplication: (outer row, inner row)
        pairs that agree on column 0 (the join's count pass; the reference's
        get_join_result_size summed, src/relation.cu:221-288)."""
        if self.kind not in ("gpu", "oracle"):
            raise GdlError(4, f"join_count is not available on the {self.kind} engine")
        out = C.c_uint64(0)
        self._call("join_count", inner.id, inner_version, outer.id, outer_version, C.byref(out))
        return int(out.value)

    def lie(self) -> Lie:
        lid = C.c_int32(-1)
        self._call("lie_create", C.byref(lid))
        return Lie(self, lid.value)

    def sync(self) -> None:
        if self.kind == "gpu":
            self._check(self.lib.gdl_engine_sync(self.h))

    def set_tuning(self, **kw) -> None:
        """Set gdl_tuning fields by name (dedup may be "auto"/"sort"/"dense")."""
        t = self.get_tuning()
        for k, v in kw.items():
            if k == "dedup" and isinstance(v, str):
                v = self.DEDUP[v]
            setattr(t, k, int(v))
        self._check(self.lib.gdl_engine_set_tuning(self.h, C.byref(t)))

    def get_tuning(self) -> Tuning:
        t = Tuning()
        self._check(self.lib.gdl_engine_get_tuning(self.h, C.byref(t)))
        return t

    def set_instances(self, node_counts) -> int:
        """Batched form: declare the instances' node counts; returns S, the
        shift of global ids (instance << S) | local."""
        counts = np.ascontiguousarray(np.asarray(node_counts, dtype=np.uint32))
        self._check(self.lib.gdl_engine_set_instances(
            self.h, counts.ctypes.data_as(C.POINTER(C.c_uint32)), len(counts)))
        if len(counts) == 0:
            return 0
        sh = C.c_int32(0)
        self._check(self.lib.gdl_engine_instance_shift(self.h, C.byref(sh)))
        return int(sh.value)

    def clear(self) -> None:
        """Drop every relation and LIE; keep buffers and the memory pool."""
        if self.kind == "gpu":
            self._check(self.lib.gdl_engine_clear(self.h))
        else:
            self._check(getattr(self.lib, self.pre + "engine_clear")(self.h))
        self.relations = []

    def test_timeout(self, polls: int) -> None:
        """The next fixpoint waits on a device flag nothing sets and gives
        up after `polls` polls: it raises GdlError(TIMEOUT); clear()
        recovers the engine (GPU engine only, for tests)."""
        self._check(self.lib.gdl_engine_test_timeout(self.h, int(polls)))

    def load_device(self, rel: Relation, ptr: int, n_rows: int) -> None:
        """load_relation from rows already in device memory (n_rows x 2 u64)."""
        self._check(self.lib.gdl_relation_load_device(self.h, rel.id, C.c_void_p(ptr), n_rows))

    def export_device(self, rel: Relation, version: int, ptr: int, cap_rows: int) -> int:
        """One version's sorted rows (arity 2) into device memory at ptr
        (room for cap_rows rows of two u64); returns the row count."""
        n = C.c_uint64(0)
        self._check(self.lib.gdl_relation_export_device(self.h, rel.id, version, C.c_void_p(ptr),
                                                        cap_rows, C.byref(n)))
        return int(n.value)

    def partition_rows(self, ptr: int, n_rows: int, column: int, world: int,
                       out_ptr: int) -> list:
        """Group n_rows device rows (two u64 columns) by owner = column value
        % world into out_ptr, one block per destination in rank order;
        returns the block sizes."""
        counts = (C.c_uint64 * world)()
        self._check(self.lib.gdl_partition_rows(self.h, C.c_void_p(ptr), n_rows, column, world,
                                                C.c_void_p(out_ptr), counts))
        return [int(x) for x in counts]

    # -- per-kernel accounting (GPU only) -----------------------------------
    def set_profile(self, flag: bool) -> None:
        self._check(self.lib.gdl_engine_set_profile(self.h, int(bool(flag))))

    def profile_reset(self) -> None:
        self._check(self.lib.gdl_engine_profile_reset(self.h))

    def profile(self) -> dict:
        """{kernel family: {"launches", "ms", "bytes"}}."""
        k = self.lib.gdl_profile_kinds()
        out = (C.c_double * (3 * k))()
        self._check(self.lib.gdl_engine_profile(self.h, out, 3 * k))
        res = {}
        for i in range(k):
            name = self.lib.gdl_profile_kind_name(i).decode()
            res[name] = {"launches": int(out[3 * i]), "ms": out[3 * i + 1],
                         "bytes": int(out[3 * i + 2])}
        return res


def digest_rows(rows: np.ndarray) -> int:
    """Host restatement of gdl_relation_digest over already-sorted rows."""
    M = (1 << 64) - 1

    def mix(x):
        x = (x + 0x9E3779B97F4A7C15) & M
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
        return x ^ (x >> 31)

    s = 0
    for i, row in enumerate(rows.tolist()):
        h = mix(i)
        for c in row:
            h = mix(h ^ c)
        s = (s + h) & M
    return mix(s ^ len(rows))
