"""GPU parity of DPsize (gpuqo_algorithm = dpsize) against the reference.

tests/golden/dpsize_cases.jsonl holds the plans of the reference's
cpu_dpsize (gpuqo_cpu_dpsize.cu): level lists built join size by join size,
left size from large to small, each pair costed in list order, the first
strict minimum kept, the level-1 list in the order of the reference's hash
memo and later lists in discovery order.  The library's GPU DPsize must
return those plans bit for bit (ties included) for the three DPsize codes
(GPUQO_DPSIZE, GPUQO_CPU_DPSIZE, GPUQO_DPE_DPSIZE), alone, inside IDP2, in a
batch call and through the serving loop.
"""
import json
import os

import pytest

from conftest import REPO, same_tree

import harness
from gpuqo_b200 import capi, lib
from gpuqo_b200.query import Query

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(REPO, "tests", "golden", "dpsize_cases.jsonl")
CODES = (capi.GPUQO_DPSIZE, capi.GPUQO_CPU_DPSIZE, capi.GPUQO_DPE_DPSIZE)


def _load():
    out = []
    with open(GOLDEN) as f:
        for line in f:
            rec = json.loads(line)
            rec["query"] = Query.from_dict(rec["query"])
            out.append(rec)
    return out


CASES = _load()


@pytest.mark.parametrize("case", CASES, ids=[f'{c["tag"]}-{c["name"]}' for c in CASES])
def test_dpsize_golden(case):
    for code in CODES:
        r = lib.run(case["query"], code, idp_n_iters=case["idp_n_iters"], idp_type=case["idp_type"])
        assert r.error == 0, (code, r.error)
        assert same_tree(r.tree, case["expected"]), code


def test_dpsize_same_optimum_as_dpsub():
    """Both searches cover every csg-cmp pair, so the root costs agree; not
    always bit for bit: where two splits of a set tie on total cost, DPsize
    and DPsub may keep different ones (different startup cost or rows), and
    the costs above them then differ in the last bits.  Tolerance: 1e-6
    relative."""
    for c in CASES:
        if c["idp_n_iters"]:
            continue
        a = lib.run(c["query"], capi.GPUQO_DPSIZE)
        b = lib.run(c["query"], capi.GPUQO_CPU_DPSUB)
        assert a.error == 0 and b.error == 0
        x, y = a.tree[3], b.tree[3]
        assert (x != x and y != y) or abs(x - y) <= 1e-6 * max(abs(x), abs(y)), c["name"]


def test_dpsize_batch_and_server():
    exact = [c for c in CASES if c["idp_n_iters"] == 0]
    trees, rc = lib.run_batch([c["query"] for c in exact], capi.GPUQO_DPSIZE)
    assert rc == 0
    for t, c in zip(trees, exact):
        assert same_tree(t, c["expected"]), c["name"]
    srv = lib.Server(max_inflight=4, wave_memory_mb=2048)
    try:
        tickets = [srv.submit(c["query"], capi.GPUQO_DPSIZE, idp_n_iters=c["idp_n_iters"],
                              idp_type=c["idp_type"]) for c in CASES]
        for tk, c in zip(tickets, CASES):
            rc, tree, _ = srv.wait(tk)
            assert rc == 0 and same_tree(tree, c["expected"]), c["name"]
    finally:
        srv.stop()


@pytest.mark.skipif(not harness.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", range(4))
def test_dpsize_vs_reference_live(seed):
    from gpuqo_b200 import query
    qs = [query.random_graph(9 + seed, 9700 + seed, extra_edge_p=0.25, rich=True),
          query.random_graph(10 + seed, 9710 + seed, equal=True),
          query.snowflake(13 + seed, 9720 + seed), query.cycle(8 + seed, 9730 + seed)]
    for q in qs:
        want, _ = harness.run_ref(q, capi.GPUQO_CPU_DPSIZE)
        got = lib.run(q, capi.GPUQO_DPSIZE)
        assert got.error == 0 and same_tree(got.tree, want), q.name
