"""CPU tests of the oracle: the plain-C restatement against the golden
fixtures (generated from the reference's own code) and, where the reference
library is built, against the reference directly."""
import pytest

from conftest import load_golden, same_tree

import harness
from gpuqo_b200 import query


GOLDEN = load_golden()
# cases the plain-C port replays in seconds; the 18-relation clique (3^18
# candidate splits, half an hour of single-threaded CPU) is checked against the
# GPU only, the port's clique cases stop at 14 relations
PORT_CASES = [c for c in GOLDEN if c["query"].n <= 20 and c["tag"] != "clique18"]


@pytest.mark.parametrize("case", PORT_CASES, ids=[f'{c["tag"]}-{c["name"]}-a{c["algorithm"]}' for c in PORT_CASES])
def test_port_matches_golden(case):
    tree, _ = harness.run_port(case["query"], case["algorithm"])
    assert same_tree(tree, case["expected"])


@pytest.mark.parametrize("tag", ["snowflake25"])
def test_port_matches_golden_full_size(tag):
    cases = [c for c in GOLDEN if c["tag"] == tag]
    assert cases
    for c in cases[:1]:
        tree, _ = harness.run_port(c["query"], c["algorithm"])
        assert same_tree(tree, c["expected"])


@pytest.mark.skipif(not harness.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", range(6))
def test_port_matches_reference_random(seed):
    qs = [query.random_graph(7 + seed, 100 + seed, extra_edge_p=0.3, rich=True),
          query.random_graph(9, 200 + seed, equal=True),
          query.cycle(9 + seed, 300 + seed),
          query.snowflake(11 + seed, 400 + seed, rich=True)]
    for q in qs:
        for alg in (3, 5):
            r, _ = harness.run_ref(q, alg)
            p, _ = harness.run_port(q, alg)
            assert same_tree(r, p), (q.name, alg)


def test_golden_covers_configs():
    tags = {c["tag"] for c in GOLDEN}
    for t in ("star12", "snowflake25", "clique10", "chain20", "cycle20", "equal_ties", "multi_member"):
        assert t in tags


def test_generators_deterministic():
    a = query.snowflake(25, 7).to_json()
    b = query.snowflake(25, 7).to_json()
    assert a == b
    q = query.snowflake(25, 7)
    assert q.n == 25 and len(q.eq_classes) == 24
    # connected, tree-shaped
    assert sum(len(e) for e in q.edges) == 2 * 24


# the sparse driver (hash memo over the connected sets): the oracle at 29 to 63
# relations, pinned to the reference's plans below that
SPARSE_PIN = ([c for c in GOLDEN if c["query"].n <= 14 and not c["tag"].startswith("clique")][:40] +
              [c for c in GOLDEN if c["tag"] in ("chain30", "cycle30", "chain30_bicc", "cycle30_bicc", "clique10")] +
              [c for c in GOLDEN if c["tag"] == "snowflake25"][:1])


@pytest.fixture
def sparse_from():
    import ctypes as C
    lib = harness.load_port()
    v = C.c_int.in_dll(lib, "oracle_sparse_from_rels")
    old = v.value
    yield lambda x: setattr(v, "value", x)
    v.value = old


def test_sparse_driver_matches_golden(sparse_from):
    sparse_from(2)
    for c in SPARSE_PIN:
        tree, _ = harness.run_port(c["query"], c["algorithm"])
        assert same_tree(tree, c["expected"]), (c["tag"], c["name"], c["algorithm"])


# the snowflakes of 32 and 34 relations (1.2 M and 2.4 M connected sets) take
# the oracle minutes; the GPU tests compare them
WIDE = [c for c in load_golden("wide_cases.jsonl") if not c["tag"].startswith("wide_snowflake")]


@pytest.mark.parametrize("case", WIDE, ids=[c["tag"] for c in WIDE])
def test_sparse_driver_reaches_reference_dpccp_optimum(case):
    """32 to 63 relations: the reference's cpu_dpccp optimum (root rows and
    total cost) is what the oracle's DPsub and MPDP reach."""
    ref = case["expected"]
    for alg in (3, 5):
        tree, _ = harness.run_port(case["query"], alg)
        assert tree is not None
        assert (tree[1], tree[3]) == (ref[1], ref[3]), (alg, tree[1:4], ref[1:4])
