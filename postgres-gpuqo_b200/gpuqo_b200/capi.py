"""ctypes view of the reference's C ABI for the join-order DP path.

The structures mirror, field for field, the reference's C headers so that the
same bytes can be handed to any library exporting ``gpuqo_run``:

* ``Bitmapset`` - Postgres nodes/bitmapset.h (``nwords`` + 64-bit words),
  as re-declared by src/backend/optimizer/gpuqo/gpuqo_postgres.cuh:29-33;
* ``PathCost``, ``GpuqoIndexInfo``, ``VarStats``, ``VarInfo`` -
  src/include/optimizer/gpuqo_common.h:92-120;
* ``EqClassInfo``, ``BaseRelationC``, ``GpuqoPlannerInfoC``, ``QueryTreeC`` -
  src/include/optimizer/gpuqo_planner_info.h:163-198.

``PlannerInfoBuilder`` turns a :class:`~gpuqo_b200.query.Query` into a
``GpuqoPlannerInfoC`` the way the planner glue does (gpuqo_main.c:549-584):
relation i gets the relid bit i+1, edges and equivalence classes become
Bitmapsets, and the equivalence classes form a linked list.  The builder owns
every buffer (the callee borrows them, as in the reference).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Tuple

from .query import Query

bitmapword = C.c_uint64


class PathCost(C.Structure):
    _fields_ = [("startup", C.c_float), ("total", C.c_float)]


class GpuqoIndexInfo(C.Structure):
    _fields_ = [("available", C.c_bool), ("unique", C.c_bool),
                ("rows", C.c_float), ("cost", PathCost)]


class VarStats(C.Structure):
    _fields_ = [("stadistinct", C.c_float), ("stanullfrac", C.c_float),
                ("mcvfreq", C.c_float)]


class VarInfoC(C.Structure):
    _fields_ = [("stats", VarStats), ("index", GpuqoIndexInfo)]


class BitmapsetHdr(C.Structure):
    _fields_ = [("nwords", C.c_int)]


class EqClassInfo(C.Structure):
    pass


EqClassInfo._fields_ = [("eclass", C.c_void_p), ("relids", C.c_void_p),
                        ("sels", C.POINTER(C.c_float)),
                        ("vars", C.POINTER(VarInfoC)),
                        ("fk", C.POINTER(C.c_void_p)),
                        ("next", C.POINTER(EqClassInfo))]


class BaseRelationC(C.Structure):
    _fields_ = [("id", C.c_void_p), ("rows", C.c_float), ("tuples", C.c_float),
                ("cost", PathCost), ("width", C.c_int)]


class GpuqoPlannerInfoC(C.Structure):
    _fields_ = [("n_rels", C.c_int),
                ("base_rels", C.POINTER(BaseRelationC)),
                ("edge_table", C.POINTER(C.c_void_p)),
                ("eq_classes", C.POINTER(EqClassInfo)),
                ("n_eq_classes", C.c_int), ("n_eq_class_sels", C.c_int),
                ("n_eq_class_fks", C.c_int), ("n_eq_class_vars", C.c_int)]


class QueryTreeC(C.Structure):
    pass


QueryTreeC._fields_ = [("id", C.c_void_p), ("rows", C.c_float),
                       ("cost", PathCost), ("width", C.c_int),
                       ("left", C.POINTER(QueryTreeC)),
                       ("right", C.POINTER(QueryTreeC))]


# GpuqoAlgorithm (src/include/optimizer/gpuqo_common.h:13-29)
GPUQO_DPSIZE = 0
GPUQO_DPSUB = 1
GPUQO_CPU_DPSIZE = 2
GPUQO_CPU_DPSUB = 3
GPUQO_CPU_DPSUB_PARALLEL = 4
GPUQO_CPU_DPSUB_BICC = 5
GPUQO_CPU_DPSUB_BICC_PARALLEL = 6
GPUQO_CPU_DPCCP = 7
GPUQO_DPE_DPSIZE = 8
GPUQO_DPE_DPSUB = 9
GPUQO_DPE_DPCCP = 10
GPUQO_CPU_GOO = 11

# GpuqoIDPType (gpuqo_common.h:31-36)
GPUQO_IDP1 = 0
GPUQO_IDP2 = 1
GPUQO_UNION = 2


def make_bitmapset(bits: int):
    """A Postgres Bitmapset holding the given Python-int bit mask."""
    nwords = max(1, (bits.bit_length() + 63) // 64)
    buf = (C.c_uint64 * (nwords + 1))()
    # header: int nwords, padded to 8 bytes (words[] is 8-aligned)
    C.cast(buf, C.POINTER(C.c_int))[0] = nwords
    for w in range(nwords):
        buf[1 + w] = (bits >> (64 * w)) & 0xFFFFFFFFFFFFFFFF
    return buf


def read_bitmapset(ptr: int) -> int:
    if not ptr:
        return 0
    nwords = C.cast(ptr, C.POINTER(C.c_int))[0]
    words = C.cast(ptr + 8, C.POINTER(C.c_uint64))
    v = 0
    for w in range(nwords):
        v |= int(words[w]) << (64 * w)
    return v


class PlannerInfoBuilder:
    """Owns the ctypes buffers of one GpuqoPlannerInfoC."""

    def __init__(self, q: Query):
        self.q = q
        self._keep: List = []
        n = q.n
        self.base = (BaseRelationC * n)()
        for i in range(n):
            bms = self._bms(1 << (i + 1))
            br = self.base[i]
            br.id = C.addressof(bms)
            br.rows = q.rows[i]
            br.tuples = q.tuples[i]
            br.cost = PathCost(q.startup[i], q.total[i])
            br.width = q.width[i]
        self.edges = (C.c_void_p * n)()
        for i, m in enumerate(q.edge_masks()):
            self.edges[i] = C.addressof(self._bms(m)) if m else None
        self.ecs = (EqClassInfo * max(1, len(q.eq_classes)))()
        n_sels = n_fks = 0
        for k, ec in enumerate(q.eq_classes):
            s = len(ec.members)
            mask = 0
            for m in ec.members:
                mask |= 1 << (m + 1)
            e = self.ecs[k]
            e.eclass = None
            e.relids = C.addressof(self._bms(mask))
            sels = (C.c_float * max(1, len(ec.sels)))(*ec.sels)
            self._keep.append(sels)
            e.sels = C.cast(sels, C.POINTER(C.c_float))
            vars_ = (VarInfoC * s)()
            for j, v in enumerate(ec.vars):
                vars_[j].stats = VarStats(v.stadistinct, v.stanullfrac, v.mcvfreq)
                vars_[j].index = GpuqoIndexInfo(v.index_available, v.index_unique,
                                                v.index_rows,
                                                PathCost(v.index_startup, v.index_total))
            self._keep.append(vars_)
            e.vars = C.cast(vars_, C.POINTER(VarInfoC))
            fk = (C.c_void_p * s)()
            for j, targets in enumerate(ec.fks):
                if targets:
                    fm = 0
                    for t in targets:
                        fm |= 1 << (t + 1)
                    fk[j] = C.addressof(self._bms(fm))
                else:
                    fk[j] = None
            self._keep.append(fk)
            e.fk = C.cast(fk, C.POINTER(C.c_void_p))
            n_sels += len(ec.sels)
            n_fks += s
        for k in range(len(q.eq_classes)):
            if k + 1 < len(q.eq_classes):
                self.ecs[k].next = C.pointer(self.ecs[k + 1])
            else:
                self.ecs[k].next = None
        self.info = GpuqoPlannerInfoC()
        self.info.n_rels = n
        self.info.base_rels = C.cast(self.base, C.POINTER(BaseRelationC))
        self.info.edge_table = C.cast(self.edges, C.POINTER(C.c_void_p))
        self.info.eq_classes = (C.pointer(self.ecs[0]) if q.eq_classes
                                else C.POINTER(EqClassInfo)())
        self.info.n_eq_classes = len(q.eq_classes)
        self.info.n_eq_class_sels = n_sels
        self.info.n_eq_class_fks = n_fks
        self.info.n_eq_class_vars = n_fks

    def _bms(self, bits):
        b = make_bitmapset(bits)
        self._keep.append(b)
        return b

    def pointer(self):
        return C.pointer(self.info)


def tree_to_py(ptr) -> Optional[tuple]:
    """QueryTreeC* -> (relid_mask, rows, startup, total, width, left, right)
    with Postgres relid bits (relation i is bit i+1)."""
    if not ptr:
        return None
    t = ptr.contents
    return (read_bitmapset(t.id), t.rows, t.cost.startup, t.cost.total,
            t.width, tree_to_py(t.left), tree_to_py(t.right))


def bind_gpuqo_run(lib):
    f = lib.gpuqo_run
    f.restype = C.POINTER(QueryTreeC)
    f.argtypes = [C.c_int, C.POINTER(GpuqoPlannerInfoC)]
    return f


def set_int(lib, name: str, value: int):
    C.c_int.in_dll(lib, name).value = int(value)


def set_bool(lib, name: str, value: bool):
    C.c_bool.in_dll(lib, name).value = bool(value)


def get_int(lib, name: str) -> int:
    return C.c_int.in_dll(lib, name).value


def same_plan(a, b) -> bool:
    """Two plans from tree_to_py are identical: relids, float32 bits of rows,
    startup and total cost (any NaN equals any NaN: payloads differ between
    x86 and GPU arithmetic, and Postgres never inspects them), width, shape."""
    import math
    import struct
    if a is None or b is None:
        return a is None and b is None

    def same_f(x, y):
        if math.isnan(x) or math.isnan(y):
            return math.isnan(x) and math.isnan(y)
        return struct.pack("<f", x) == struct.pack("<f", y)
    return (a[0] == b[0] and a[4] == b[4] and all(same_f(a[i], b[i]) for i in (1, 2, 3))
            and same_plan(a[5], b[5]) and same_plan(a[6], b[6]))
