"""Loaders for the two CPU oracles (TEST INFRASTRUCTURE ONLY).

* ``oracle/_ref/libgpuqo_ref.so`` - the reference's own gpuqo module compiled
  from its sources (oracle/Makefile target ``ref``).  Its ``gpuqo_run`` with
  GPUQO_CPU_DPSUB / GPUQO_CPU_DPSUB_BICC is the parity contract; its
  GPUQO_CPU_DPSUB_BICC_PARALLEL and GPUQO_DPE_DPSUB are the timed CPU
  baselines.
* ``oracle/libgpuqo_oracle.so`` - the plain-C restatement (gpuqo_oracle.c),
  pinned against the reference library and the golden fixtures.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PKG = os.path.join(REPO, "postgres-gpuqo_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)

from gpuqo_b200 import capi  # noqa: E402
from gpuqo_b200.query import Query  # noqa: E402

REF_SO = os.path.join(HERE, "_ref", "libgpuqo_ref.so")
# the same sources built for the build machine's CPU (-march=native): a
# separately reported CPU-baseline flavour, never the parity oracle
REF_NATIVE_SO = os.path.join(HERE, "_ref", "libgpuqo_ref_native.so")
PORT_SO = os.path.join(HERE, "libgpuqo_oracle.so")

_ref = {}
_port = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def load_ref(native=False):
    """The reference library, with the GUC globals it needs initialised
    (they are zero in a bare process; gpuqo_cpu_dpe.cu:33-34 and
    gpuqo_cpu_dpsub_parallel.cu:30 read them)."""
    if native not in _ref:
        lib = C.CDLL(REF_NATIVE_SO if native else REF_SO, mode=C.RTLD_LOCAL)
        capi.bind_gpuqo_run(lib)
        lib.ref_free_query_tree.argtypes = [C.c_void_p]
        lib.ref_free_query_tree.restype = None
        capi.set_int(lib, "gpuqo_dpe_n_threads", os.cpu_count() or 1)
        capi.set_int(lib, "gpuqo_cpu_dpsub_parallel_chunk_size", 256)
        capi.set_int(lib, "gpuqo_dpe_pairs_per_depbuf", 65536)
        capi.set_int(lib, "gpuqo_idp_n_iters", 0)
        capi.set_int(lib, "gpuqo_idp_type", capi.GPUQO_IDP2)
        capi.set_bool(lib, "gpuqo_spanning_tree_enable", False)
        _ref[native] = lib
    return _ref[native]


def load_port():
    global _port
    if _port is None:
        lib = C.CDLL(PORT_SO, mode=C.RTLD_LOCAL)
        capi.bind_gpuqo_run(lib)
        lib.oracle_free_query_tree.argtypes = [C.c_void_p]
        lib.oracle_free_query_tree.restype = None
        _port = lib
    return _port


def _silence():
    """The reference prints progress lines from IDP drivers; route fd 1 to
    /dev/null for the duration of a call."""
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    os.close(devnull)
    return saved


def _restore(saved):
    try:
        C.CDLL(None).fflush(None)
    except Exception:
        pass
    os.dup2(saved, 1)
    os.close(saved)


def run_ref(q: Query, algorithm: int, idp_n_iters: int = 0,
            idp_type: int = capi.GPUQO_IDP2, threads: int = 0, quiet=True, native=False, spanning=False):
    """Run the reference's gpuqo_run; returns (tree, seconds).  spanning sets
    gpuqo_spanning_tree_enable for the call."""
    lib = load_ref(native)
    capi.set_int(lib, "gpuqo_idp_n_iters", idp_n_iters)
    capi.set_int(lib, "gpuqo_idp_type", idp_type)
    capi.set_bool(lib, "gpuqo_spanning_tree_enable", spanning)
    if threads:
        capi.set_int(lib, "gpuqo_dpe_n_threads", threads)
    b = capi.PlannerInfoBuilder(q)
    saved = _silence() if quiet else None
    try:
        t0 = time.perf_counter()
        res = lib.gpuqo_run(algorithm, b.pointer())
        dt = time.perf_counter() - t0
    finally:
        if saved is not None:
            _restore(saved)
    tree = capi.tree_to_py(res)
    lib.ref_free_query_tree(C.cast(res, C.c_void_p))
    return tree, dt


def run_port(q: Query, algorithm: int, idp_n_iters: int = 0,
             idp_type: int = capi.GPUQO_IDP2):
    lib = load_port()
    capi.set_int(lib, "gpuqo_idp_n_iters", idp_n_iters)
    capi.set_int(lib, "gpuqo_idp_type", idp_type)
    b = capi.PlannerInfoBuilder(q)
    t0 = time.perf_counter()
    res = lib.gpuqo_run(algorithm, b.pointer())
    dt = time.perf_counter() - t0
    tree = capi.tree_to_py(res)
    lib.oracle_free_query_tree(C.cast(res, C.c_void_p))
    return tree, dt


def eval_join(q: Query, left_id: int, right_id: int, lvals, rvals):
    """Oracle join evaluation (rows, startup, total, width) of one join
    (queries of at most 63 relations, the oracle's relation sets)."""
    if q.n > 63:
        raise ValueError(f"the oracle takes at most 63 relations, not {q.n}")
    lib = load_port()
    f = lib.oracle_eval_join
    f.argtypes = [C.POINTER(capi.GpuqoPlannerInfoC), C.c_uint64, C.c_uint64,
                  C.POINTER(C.c_float), C.POINTER(C.c_float)]
    f.restype = None
    b = capi.PlannerInfoBuilder(q)
    vin = (C.c_float * 8)(*(list(lvals) + list(rvals)))
    vout = (C.c_float * 4)()
    f(b.pointer(), left_id, right_id, vin, vout)
    return tuple(vout)
