"""GPU parity of the IDP2 and UnionDP drivers (gpuqo_idp_n_iters /
gpuqo_idp_type) against the reference: golden fixtures
(tests/golden/idp_cases.jsonl) and, where the reference library is present,
live comparisons on further seeds.  Sub-problems run as MPDP on the GPU; the
reference solves them with cpu_dpsub_bicc."""
import json
import os

import pytest

from conftest import REPO, same_tree

import harness
from gpuqo_b200 import capi, lib, query
from gpuqo_b200.query import Query

pytestmark = pytest.mark.gpu

IDP_GOLDEN = os.path.join(REPO, "tests", "golden", "idp_cases.jsonl")


def _load():
    out = []
    with open(IDP_GOLDEN) as f:
        for line in f:
            rec = json.loads(line)
            rec["query"] = Query.from_dict(rec["query"])
            out.append(rec)
    return out


CASES = _load()


@pytest.mark.parametrize("case", CASES, ids=[f'{c["tag"]}-{c["name"]}-k{c["idp_n_iters"]}' for c in CASES])
def test_idp_golden(case):
    r = lib.run(case["query"], capi.GPUQO_DPSUB, bicc=True, idp_n_iters=case["idp_n_iters"],
                idp_type=case["idp_type"])
    assert r.error == 0, r.error
    assert same_tree(r.tree, case["expected"])
    assert r.stats["n_subproblems"] >= 1


@pytest.mark.skipif(not harness.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", range(4))
def test_idp_vs_reference_live(seed):
    cases = [(query.snowflake(33 + 7 * seed, 500 + seed), 11, capi.GPUQO_IDP2),
             (query.snowflake(36 + 5 * seed, 600 + seed, rich=True), 13, capi.GPUQO_UNION),
             (query.random_graph(30 + seed, 700 + seed, extra_edge_p=0.04), 9, capi.GPUQO_IDP2),
             (query.random_graph(28 + seed, 800 + seed, extra_edge_p=0.04), 9, capi.GPUQO_UNION),
             (query.star(26 + seed, 900 + seed), 8, capi.GPUQO_IDP2)]
    for q, k, typ in cases:
        want, _ = harness.run_ref(q, 5, idp_n_iters=k, idp_type=typ)
        got = lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=typ)
        assert got.error == 0
        assert same_tree(got.tree, want), (q.name, k, typ)


def test_large_query_needs_idp():
    q = query.snowflake(70, 3)
    r = lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=0)
    assert r.tree is None and r.error == 5      # GPUQO_B200_ERR_UNSUPPORTED, as the reference returns NULL


def test_cancel_between_idp_iterations():
    """A cancel request (Postgres's InterruptPending) raised while an IDP2 run
    is in flight ends it before its next sub-problem: NULL and
    GPUQO_B200_ERR_CANCELLED, nothing left running; with the flag cleared the
    same query plans normally afterwards."""
    import ctypes as C
    import threading
    import time
    l = lib.load()
    flag = C.c_int.in_dll(l, "InterruptPending")
    q = query.snowflake(1000, 77)
    capi.set_bool(l, "gpuqo_dpsub_bicc_enable", True)
    capi.set_int(l, "gpuqo_idp_n_iters", 25)
    capi.set_int(l, "gpuqo_idp_type", capi.GPUQO_IDP2)
    b = capi.PlannerInfoBuilder(q)
    warm = l.gpuqo_run(capi.GPUQO_DPSUB, b.pointer())        # engine and device set-up
    l.gpuqo_b200_free_query_tree(C.cast(warm, C.c_void_p))
    t0 = time.perf_counter()
    full = l.gpuqo_run(capi.GPUQO_DPSUB, b.pointer())        # uncancelled, for its duration
    full_s = time.perf_counter() - t0
    assert full
    want = capi.tree_to_py(full)
    l.gpuqo_b200_free_query_tree(C.cast(full, C.c_void_p))
    out = {}

    def run():
        out["tree"] = l.gpuqo_run(capi.GPUQO_DPSUB, b.pointer())   # ctypes releases the GIL
        out["err"] = l.gpuqo_b200_last_error()
    try:
        th = threading.Thread(target=run)
        th.start()
        time.sleep(full_s / 4)
        flag.value = 1
        th.join(timeout=60)
        assert not th.is_alive()
    finally:
        flag.value = 0
    assert not out["tree"] and out["err"] == 6          # GPUQO_B200_ERR_CANCELLED
    again = lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=25, idp_type=capi.GPUQO_IDP2)
    capi.set_int(l, "gpuqo_idp_n_iters", 0)
    assert again.error == 0 and same_tree(again.tree, want)
