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
