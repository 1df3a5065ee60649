"""GPU parity of gpuqo_spanning_tree_enable against the reference.

With the setting on, the reference replaces the join graph by its minimum
spanning tree (grown from relation 0 by the fewest estimated join rows)
before any algorithm runs, keeps every equivalence class for the costs, and
plans the tree (gpuqo_main_internal.cu:94-100, gpuqo_spanning_tree.cu:19-72).
tests/golden/spanning_cases.jsonl holds the plans the reference's own engines
returned with it on (exact DPsub / MPDP, IDP2 and UnionDP, 64-bit and
dynamic relation sets); the library must return them bit for bit, through
gpuqo_run, the batch entry and the serving loop.
"""
import json
import os

import pytest

from conftest import REPO, same_tree

from gpuqo_b200 import capi, lib
from gpuqo_b200.query import Query

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(REPO, "tests", "golden", "spanning_cases.jsonl")


def _load():
    out = []
    with open(GOLDEN) as f:
        for line in f:
            rec = json.loads(line)
            rec["query"] = Query.from_dict(rec["query"])
            out.append(rec)
    return out


CASES = _load()


@pytest.fixture
def spanning():
    L = lib.load()
    capi.set_bool(L, "gpuqo_spanning_tree_enable", True)
    yield
    capi.set_bool(L, "gpuqo_spanning_tree_enable", False)


@pytest.mark.parametrize("case", CASES, ids=[f'{c["tag"]}-{c["name"]}' for c in CASES])
def test_spanning_tree_golden(case, spanning):
    r = lib.run(case["query"], capi.GPUQO_DPSUB, bicc=(case["algorithm"] == 5),
                idp_n_iters=case["idp_n_iters"], idp_type=case["idp_type"])
    assert r.error == 0, r.error
    assert same_tree(r.tree, case["expected"])


def test_spanning_tree_batch_and_server(spanning):
    exact = [c for c in CASES if c["idp_n_iters"] == 0 and c["algorithm"] == 5]
    trees, rc = lib.run_batch([c["query"] for c in exact], capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    for t, c in zip(trees, exact):
        assert same_tree(t, c["expected"]), c["name"]
    srv = lib.Server(max_inflight=4, wave_memory_mb=2048)
    try:
        tickets = [srv.submit(c["query"], capi.GPUQO_DPSUB, bicc=(c["algorithm"] == 5),
                              idp_n_iters=c["idp_n_iters"], idp_type=c["idp_type"]) for c in CASES]
        for tk, c in zip(tickets, CASES):
            rc, tree, _ = srv.wait(tk)
            assert rc == 0 and same_tree(tree, c["expected"]), c["name"]
    finally:
        srv.stop()


def test_spanning_tree_off_plans_the_graph_as_given():
    """The setting off (the default) plans the original graph: on graphs with
    cycles the plan generally differs from the spanning tree's."""
    differ = 0
    for c in CASES:
        if c["idp_n_iters"]:
            continue
        r = lib.run(c["query"], capi.GPUQO_DPSUB, bicc=(c["algorithm"] == 5))
        assert r.error == 0
        differ += 0 if same_tree(r.tree, c["expected"]) else 1
    assert differ > 0
