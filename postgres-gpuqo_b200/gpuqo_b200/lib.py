"""ctypes binding of libgpuqo_b200.so (the product library).

Everything here calls through the C ABI declared in include/gpuqo_b200.h:
``gpuqo_run`` with the reference's ``GpuqoPlannerInfoC`` / ``QueryTreeC``
structures and GUC variables, plus the library's extension entry points.
There is no fallback: if the shared library is missing the import of
:func:`load` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import Dict, List, Optional

from . import capi
from .query import Query

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpuqo_b200.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "gpuqo_b200.h")


class Stats(C.Structure):
    _fields_ = [("connected_sets", C.c_uint64), ("evaluated_pairs", C.c_uint64),
                ("filtered_subsets", C.c_uint64), ("memo_bytes", C.c_uint64),
                ("device_ms", C.c_double), ("eval_kernel_ms", C.c_double),
                ("eval_kernel_launches", C.c_uint32), ("n_subproblems", C.c_uint32),
                ("kernel_launches", C.c_uint32), ("fallback_sets", C.c_uint32),
                ("barrier_timeouts", C.c_uint32), ("handoff_device_ms", C.c_double)]

    def to_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

# GUC variables whose values load() records as the library was loaded, before
# any caller changed them (boot_gucs)
_BOOT_INTS = ("gpuqo_n_parallel", "gpuqo_dpsub_filter_threshold", "gpuqo_idp_type", "gpuqo_idp_n_iters")
_BOOT_BOOLS = ("gpuqo_dpsub_ccc_enable", "gpuqo_dpsub_bicc_enable", "gpuqo_dpsub_csg_enable")
boot_gucs = {}


def load():
    """Load the product library (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build it with `make -C postgres-gpuqo_b200`")
        lib = C.CDLL(LIB_PATH, mode=C.RTLD_LOCAL)
        for name in _BOOT_INTS:
            boot_gucs[name] = C.c_int.in_dll(lib, name).value
        for name in _BOOT_BOOLS:
            boot_gucs[name] = C.c_bool.in_dll(lib, name).value
        capi.bind_gpuqo_run(lib)
        lib.gpuqo_b200_free_query_tree.argtypes = [C.c_void_p]
        lib.gpuqo_b200_free_query_tree.restype = None
        lib.gpuqo_b200_last_error.argtypes = []
        lib.gpuqo_b200_last_error.restype = C.c_int
        lib.gpuqo_b200_get_stats.argtypes = [C.POINTER(Stats)]
        lib.gpuqo_b200_get_stats.restype = None
        lib.gpuqo_b200_run_batch.argtypes = [C.c_int, C.POINTER(C.POINTER(capi.GpuqoPlannerInfoC)),
                                             C.c_int, C.POINTER(C.POINTER(capi.QueryTreeC))]
        lib.gpuqo_b200_run_batch.restype = C.c_int
        lib.gpuqo_b200_time_resident.argtypes = [C.c_int, C.POINTER(capi.GpuqoPlannerInfoC), C.c_int, C.c_int,
                                                 C.c_int, C.POINTER(C.c_double),
                                                 C.POINTER(C.POINTER(capi.QueryTreeC))]
        lib.gpuqo_b200_time_resident.restype = C.c_int
        lib.gpuqo_b200_server_start.argtypes = [C.c_int, C.c_int]
        lib.gpuqo_b200_server_start.restype = C.c_int
        lib.gpuqo_b200_server_submit.argtypes = [C.c_int, C.POINTER(capi.GpuqoPlannerInfoC), C.POINTER(C.c_uint64)]
        lib.gpuqo_b200_server_submit.restype = C.c_int
        lib.gpuqo_b200_server_wait.argtypes = [C.c_uint64, C.POINTER(C.POINTER(capi.QueryTreeC)),
                                               C.POINTER(C.c_double)]
        lib.gpuqo_b200_server_wait.restype = C.c_int
        lib.gpuqo_b200_server_stats.argtypes = [C.c_void_p]
        lib.gpuqo_b200_server_stats.restype = C.c_int
        lib.gpuqo_b200_server_stop.argtypes = []
        lib.gpuqo_b200_server_stop.restype = C.c_int
        lib.gpuqo_b200_server_cancel.argtypes = [C.c_uint64]
        lib.gpuqo_b200_server_cancel.restype = C.c_int
        lib.gpuqo_b200_reset_persistent.argtypes = []
        lib.gpuqo_b200_reset_persistent.restype = C.c_int
        _lib = lib
    return _lib


def declared_symbols() -> List[str]:
    """Function and variable names declared in include/gpuqo_b200.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    funcs = re.findall(r"^\s*(?:QueryTreeC\s*\*\s*|int\s+|void\s+)(\w+)\s*\(", text, flags=re.M)
    vars_ = re.findall(r"^\s*extern\s+(?:int|bool)\s+(\w+)\s*;", text, flags=re.M)
    return sorted(set(funcs + vars_))


def set_gucs(**gucs):
    lib = load()
    for k, v in gucs.items():
        if isinstance(v, bool):
            capi.set_bool(lib, k, v)
        else:
            capi.set_int(lib, k, v)


class RunResult:
    def __init__(self, tree, stats: Dict, error: int, seconds: float):
        self.tree = tree
        self.stats = stats
        self.error = error
        self.seconds = seconds


def run(q: Query, algorithm: int = capi.GPUQO_DPSUB, bicc: Optional[bool] = None,
        ccc: Optional[bool] = None, idp_n_iters: int = 0,
        idp_type: int = capi.GPUQO_IDP2) -> RunResult:
    """Optimise one query through gpuqo_run; returns tree + stats."""
    import time
    lib = load()
    if bicc is not None:
        capi.set_bool(lib, "gpuqo_dpsub_bicc_enable", bicc)
    if ccc is not None:
        capi.set_bool(lib, "gpuqo_dpsub_ccc_enable", ccc)
    capi.set_int(lib, "gpuqo_idp_n_iters", idp_n_iters)
    capi.set_int(lib, "gpuqo_idp_type", idp_type)
    b = capi.PlannerInfoBuilder(q)
    t0 = time.perf_counter()
    res = lib.gpuqo_run(algorithm, b.pointer())
    dt = time.perf_counter() - t0
    err = lib.gpuqo_b200_last_error()
    st = Stats()
    lib.gpuqo_b200_get_stats(C.byref(st))
    tree = capi.tree_to_py(res)
    if res:
        lib.gpuqo_b200_free_query_tree(C.cast(res, C.c_void_p))
    return RunResult(tree, st.to_dict(), err, dt)


def run_batch(queries: List[Query], algorithm: int = capi.GPUQO_DPSUB,
              bicc: Optional[bool] = None) -> (List, int):
    lib = load()
    if bicc is not None:
        capi.set_bool(lib, "gpuqo_dpsub_bicc_enable", bicc)
    capi.set_int(lib, "gpuqo_idp_n_iters", 0)
    builders = [capi.PlannerInfoBuilder(q) for q in queries]
    arr = (C.POINTER(capi.GpuqoPlannerInfoC) * len(queries))(*[b.pointer() for b in builders])
    out = (C.POINTER(capi.QueryTreeC) * len(queries))()
    rc = lib.gpuqo_b200_run_batch(algorithm, arr, len(queries), out)
    trees = []
    for i in range(len(queries)):
        trees.append(capi.tree_to_py(out[i]))
        if out[i]:
            lib.gpuqo_b200_free_query_tree(C.cast(out[i], C.c_void_p))
    return trees, rc


def time_resident(q: Query, algorithm: int = capi.GPUQO_DPSUB, bicc: Optional[bool] = None,
                  warmup: int = 3, iters: int = 10, flush_l2: bool = True):
    """Device-resident DP time (ms per replay) + the plan + stats."""
    lib = load()
    if bicc is not None:
        capi.set_bool(lib, "gpuqo_dpsub_bicc_enable", bicc)
    b = capi.PlannerInfoBuilder(q)
    ms = C.c_double(0.0)
    out = C.POINTER(capi.QueryTreeC)()
    rc = lib.gpuqo_b200_time_resident(algorithm, b.pointer(), warmup, iters, int(flush_l2), C.byref(ms),
                                      C.byref(out))
    st = Stats()
    lib.gpuqo_b200_get_stats(C.byref(st))
    tree = capi.tree_to_py(out) if rc == 0 else None
    if rc == 0 and out:
        lib.gpuqo_b200_free_query_tree(C.cast(out, C.c_void_p))
    return rc, ms.value, tree, st.to_dict()


def get_stats() -> Dict:
    lib = load()
    st = Stats()
    lib.gpuqo_b200_get_stats(C.byref(st))
    return st.to_dict()


class Tuning(C.Structure):
    _fields_ = [("single_narrow_level_sets", C.c_double), ("single_wide_level_sets", C.c_double),
                ("batch_single_sets", C.c_double), ("tune_ms", C.c_double),
                ("tuned", C.c_int)]

    def to_dict(self) -> Dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


def autotune() -> Dict:
    """Measure and install the kernel-variant and batch hand-off crossovers
    on the current device (gpuqo_b200_autotune); returns them."""
    lib = load()
    t = Tuning()
    rc = lib.gpuqo_b200_autotune(C.byref(t))
    if rc:
        raise RuntimeError(f"gpuqo_b200_autotune failed: {rc}")
    return t.to_dict()


def set_tuning(single_narrow_level_sets: float, single_wide_level_sets: float, batch_single_sets: float,
               tuned: int = 1) -> None:
    """Install crossovers without measuring (gpuqo_b200_set_tuning)."""
    lib = load()
    t = Tuning(single_narrow_level_sets, single_wide_level_sets, batch_single_sets, 0.0, tuned)
    rc = lib.gpuqo_b200_set_tuning(C.byref(t))
    if rc:
        raise ValueError(f"gpuqo_b200_set_tuning rejected {t.to_dict()}: {rc}")


def get_tuning() -> Dict:
    lib = load()
    t = Tuning()
    lib.gpuqo_b200_get_tuning(C.byref(t))
    return t.to_dict()


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("waves", C.c_uint64), ("batched_subproblems", C.c_uint64),
                ("single_subproblems", C.c_uint64), ("device_ms", C.c_double), ("busy_ms", C.c_double),
                ("starved_ms", C.c_double)]


class Server:
    """The library's continuous-batching planner service (C ABI
    gpuqo_b200_server_*).  submit() captures the GUCs current at the call."""

    def __init__(self, max_inflight: int = 16, wave_memory_mb: int = 32768):
        self.lib = load()
        rc = self.lib.gpuqo_b200_server_start(max_inflight, wave_memory_mb)
        if rc:
            raise RuntimeError(f"gpuqo_b200_server_start: {rc}")
        self._keep = {}

    def submit(self, q: Query, algorithm: int = capi.GPUQO_DPSUB, bicc: Optional[bool] = None,
               idp_n_iters: int = 0, idp_type: int = capi.GPUQO_IDP2) -> int:
        if bicc is not None:
            capi.set_bool(self.lib, "gpuqo_dpsub_bicc_enable", bicc)
        capi.set_int(self.lib, "gpuqo_idp_n_iters", idp_n_iters)
        capi.set_int(self.lib, "gpuqo_idp_type", idp_type)
        b = capi.PlannerInfoBuilder(q)
        t = C.c_uint64(0)
        rc = self.lib.gpuqo_b200_server_submit(algorithm, b.pointer(), C.byref(t))
        if rc:
            raise RuntimeError(f"gpuqo_b200_server_submit: {rc}")
        return t.value

    def submit_built(self, b: "capi.PlannerInfoBuilder", algorithm: int = capi.GPUQO_DPSUB) -> int:
        t = C.c_uint64(0)
        rc = self.lib.gpuqo_b200_server_submit(algorithm, b.pointer(), C.byref(t))
        if rc:
            raise RuntimeError(f"gpuqo_b200_server_submit: {rc}")
        return t.value

    def wait_raw(self, ticket: int):
        """gpuqo_b200_server_wait as it returns: (status, the QueryTreeC
        pointer or NULL, latency in ms); the caller frees the tree with
        gpuqo_b200_free_query_tree."""
        out = C.POINTER(capi.QueryTreeC)()
        lat = C.c_double(0.0)
        rc = self.lib.gpuqo_b200_server_wait(ticket, C.byref(out), C.byref(lat))
        return rc, out, lat.value

    def wait(self, ticket: int):
        rc, out, lat = self.wait_raw(ticket)
        tree = capi.tree_to_py(out) if (rc == 0 and out) else None
        if out:
            self.lib.gpuqo_b200_free_query_tree(C.cast(out, C.c_void_p))
        return rc, tree, lat

    def cancel(self, ticket: int) -> int:
        """Cancel one request (gpuqo_b200_server_cancel); returns the status."""
        return self.lib.gpuqo_b200_server_cancel(ticket)

    def stats(self) -> Dict:
        st = ServerStats()
        self.lib.gpuqo_b200_server_stats(C.byref(st))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def stop(self):
        self.lib.gpuqo_b200_server_stop()
