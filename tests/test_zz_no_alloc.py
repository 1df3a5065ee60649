"""GPU test of gpuqo_b200_run_noalloc, the entry point that allocates nothing.

Callers that cannot allocate device memory (a Postgres backend that must not
leak GPU memory when a cancelled query longjmps out, a process whose device
memory belongs to another pool) use this entry point; it keeps all scratch in
one static device array and therefore handles at most 18 relations.  Its plans
must be the plans gpuqo_run returns, bit for bit, on consecutive calls that
reuse the shared scratch.  This file sorts last so that a stop-at-first-failure
run has executed every other test before it.
"""
import ctypes as C

import pytest

from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu


class PlanNode(C.Structure):
    _fields_ = [("relids", C.c_uint64), ("left", C.c_int32), ("right", C.c_int32),
                ("rows", C.c_float), ("startup", C.c_float), ("total", C.c_float),
                ("width", C.c_int32)]


def _bind():
    l = lib.load()
    f = l.gpuqo_b200_run_noalloc
    f.argtypes = [C.c_int, C.POINTER(capi.GpuqoPlannerInfoC), C.c_void_p,
                  C.POINTER(PlanNode), C.c_int, C.POINTER(C.c_int)]
    f.restype = C.c_int
    return f


def _nodes_to_tree(nodes, i):
    if i < 0:
        return None
    nd = nodes[i]
    return (nd.relids, nd.rows, nd.startup, nd.total, nd.width,
            _nodes_to_tree(nodes, nd.left), _nodes_to_tree(nodes, nd.right))


def run_noalloc(q, algorithm):
    f = _bind()
    b = capi.PlannerInfoBuilder(q)
    nodes = (PlanNode * 64)()
    n_out = C.c_int(0)
    rc = f(algorithm, b.pointer(), None, nodes, 64, C.byref(n_out))
    assert rc == 0, f"gpuqo_b200_run_noalloc returned {rc}"
    assert n_out.value == 2 * q.n - 1
    return _nodes_to_tree(nodes, 0)


def test_noalloc_matches_gpuqo_run_twice():
    cases = [(query.snowflake(18, 11), capi.GPUQO_CPU_DPSUB_BICC),
             (query.cycle(14, 12), capi.GPUQO_CPU_DPSUB)]
    for q, alg in cases:
        want = lib.run(q, alg)
        assert want.error == 0 and want.tree is not None
        first = run_noalloc(q, alg)
        second = run_noalloc(q, alg)
        assert first == want.tree
        assert second == want.tree


def test_noalloc_rejects_oversized_query():
    f = _bind()
    q = query.chain(19, 0)
    b = capi.PlannerInfoBuilder(q)
    nodes = (PlanNode * 64)()
    n_out = C.c_int(0)
    rc = f(capi.GPUQO_CPU_DPSUB_BICC, b.pointer(), None, nodes, 64, C.byref(n_out))
    assert rc == 4   # GPUQO_B200_ERR_TOO_LARGE
