"""GPU test of gpuqo_b200_run_noalloc, the entry point that allocates nothing.

Callers that cannot allocate device memory (a Postgres backend that must not
leak GPU memory when a cancelled query longjmps out, a process whose device
memory belongs to another pool) use this entry point; it keeps all scratch in
one static device array and therefore handles at most 18 relations and a
planner info of at most 6144 words.  Its plans must be the plans gpuqo_run
returns, bit for bit, on consecutive calls that reuse the shared scratch.
This file sorts last so that a stop-at-first-failure run has executed every
other test before it.
"""
import ctypes as C

import pytest

from conftest import same_tree
from gpuqo_b200 import capi, lib, query
from gpuqo_b200.query import EqClass, VarInfo

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


def _call(q, algorithm):
    f = _bind()
    b = capi.PlannerInfoBuilder(q)
    nodes = (PlanNode * 64)()
    n_out = C.c_int(0)
    rc = f(algorithm, b.pointer(), None, nodes, 64, C.byref(n_out))
    return rc, nodes, n_out.value


def run_noalloc(q, algorithm):
    rc, nodes, n_out = _call(q, algorithm)
    assert rc == 0, f"gpuqo_b200_run_noalloc returned {rc}"
    assert n_out == 2 * q.n - 1
    return _nodes_to_tree(nodes, 0)


# tree-shaped, cyclic and dense graphs; column statistics and unique indexes;
# classes of three and four members; all-equal relations (cost ties); a clique
# of 13 whose largest sets take the chunked overflow path
CASES = [
    ("snowflake18", lambda: query.snowflake(18, 11), (capi.GPUQO_CPU_DPSUB_BICC,)),
    ("cycle14", lambda: query.cycle(14, 12), (capi.GPUQO_CPU_DPSUB, capi.GPUQO_CPU_DPSUB_BICC)),
    ("random_rich14", lambda: query.random_graph(14, 3, extra_edge_p=0.25, rich=True),
     (capi.GPUQO_CPU_DPSUB, capi.GPUQO_CPU_DPSUB_BICC)),
    ("multi_member12", lambda: query.multi_member_classes(12, 5), (capi.GPUQO_CPU_DPSUB, capi.GPUQO_CPU_DPSUB_BICC)),
    ("equal_ties12", lambda: query.random_graph(12, 4, equal=True), (capi.GPUQO_CPU_DPSUB, capi.GPUQO_CPU_DPSUB_BICC)),
    ("clique13", lambda: query.clique(13, 6), (capi.GPUQO_CPU_DPSUB, capi.GPUQO_CPU_DPSUB_BICC)),
]


@pytest.mark.parametrize("ccc", [True, False], ids=["ccc_on", "ccc_off"])
@pytest.mark.parametrize("name,make,algs", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_gpuqo_run_twice(name, make, algs, ccc):
    q = make()
    try:
        lib.set_gucs(gpuqo_dpsub_ccc_enable=ccc)
        for alg in algs:
            want = lib.run(q, alg)
            assert want.error == 0 and want.tree is not None
            first = run_noalloc(q, alg)
            second = run_noalloc(q, alg)
            assert same_tree(first, want.tree), (name, alg)
            assert same_tree(second, want.tree), (name, alg)
    finally:
        lib.set_gucs(gpuqo_dpsub_ccc_enable=True)


def test_noalloc_rejects_oversized_query():
    rc, _, _ = _call(query.chain(19, 0), capi.GPUQO_CPU_DPSUB_BICC)
    assert rc == 4   # GPUQO_B200_ERR_TOO_LARGE


def test_noalloc_rejects_oversized_planner_info_and_recovers():
    """Many wide classes on few relations exceed the static planner-info
    area: GPUQO_B200_ERR_TOO_LARGE, and the next call is unaffected."""
    q = query.chain(10, 1)
    members = list(range(10))
    wide = EqClass(members=members, sels=[0.5] * 45, fks=[[] for _ in members], vars=[VarInfo() for _ in members])
    q.eq_classes = q.eq_classes + [wide] * 60
    rc, _, _ = _call(q, capi.GPUQO_CPU_DPSUB_BICC)
    assert rc == 4   # GPUQO_B200_ERR_TOO_LARGE
    ok = query.snowflake(16, 2)
    want = lib.run(ok, capi.GPUQO_CPU_DPSUB_BICC)
    assert same_tree(run_noalloc(ok, capi.GPUQO_CPU_DPSUB_BICC), want.tree)
