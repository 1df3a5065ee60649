"""GPU parity: the product library (C ABI gpuqo_run on a B200) against the
reference's plans.

* golden fixtures (tests/golden/cases.jsonl, produced by the reference's own
  cpu_dpsub / cpu_dpsub_bicc) -- bit-identical trees: relids, rows, startup
  and total cost, width and shape;
* seeded random graphs against the oracle restatement (pinned to the
  reference by tests/test_oracle.py), both enumerators, CCC on and off;
* full-size cases without a CPU oracle run: every node of the plan is
  re-evaluated by the oracle's join arithmetic, and MPDP and DPsub must agree
  on the optimal root cost.
"""
import pytest

from conftest import load_golden, same_tree

import harness
from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu

GOLDEN = load_golden()
# the configurations' own workloads at their full sizes: the 25-relation
# snowflakes (MPDP), the 18-relation clique (plain DPsub), the 30-relation
# chain and cycle (both), the 14-relation clique under MPDP
FULL_SIZE_TAGS = {"snowflake25", "clique18", "clique14_bicc", "chain30", "cycle30", "chain30_bicc", "cycle30_bicc"}
FAST = [c for c in GOLDEN if c["tag"] not in FULL_SIZE_TAGS]
SLOW = [c for c in GOLDEN if c["tag"] in FULL_SIZE_TAGS]


def gpu_run(q, alg, ccc=True):
    """alg 3 -> plain DPsub, alg 5 -> MPDP, through gpuqo_algorithm=dpsub."""
    r = lib.run(q, capi.GPUQO_DPSUB, bicc=(alg == 5), ccc=ccc)
    assert r.error == 0, f"gpuqo_b200 error {r.error}"
    return r


@pytest.mark.parametrize("case", FAST, ids=[f'{c["tag"]}-{c["name"]}-a{c["algorithm"]}' for c in FAST])
def test_golden(case):
    r = gpu_run(case["query"], case["algorithm"])
    assert same_tree(r.tree, case["expected"])


@pytest.mark.parametrize("case", SLOW, ids=[f'{c["tag"]}-{c["name"]}-a{c["algorithm"]}' for c in SLOW])
def test_golden_full_size(case):
    r = gpu_run(case["query"], case["algorithm"])
    assert same_tree(r.tree, case["expected"])


@pytest.mark.parametrize("case", [c for c in FAST if c["tag"] in ("star12", "random_rich")][:6])
def test_cpu_algorithm_codes(case):
    """GPUQO_CPU_DPSUB / GPUQO_CPU_DPSUB_BICC codes return the same plans."""
    r = lib.run(case["query"], case["algorithm"])
    assert r.error == 0
    assert same_tree(r.tree, case["expected"])


@pytest.mark.parametrize("seed", range(12))
def test_random_vs_oracle(seed):
    qs = [query.random_graph(5 + seed % 10, 1000 + seed, extra_edge_p=0.3, rich=(seed % 2 == 0)),
          query.random_graph(10, 2000 + seed, equal=True),
          query.cycle(6 + seed, 3000 + seed),
          query.clique(4 + seed % 6, 4000 + seed, rich=True),
          query.snowflake(12 + seed % 6, 5000 + seed),
          query.multi_member_classes(7 + seed % 5, 6000 + seed)]
    for q in qs:
        for alg in (3, 5):
            want, _ = harness.run_port(q, alg)
            for ccc in (True, False):
                got = gpu_run(q, alg, ccc=ccc)
                assert same_tree(got.tree, want), (q.name, alg, ccc)


@pytest.mark.parametrize("seed", range(6))
def test_tree_queries_with_ties(seed):
    """Tree-shaped queries take the tree kernel; all-equal relations make
    most costs tie, so most sets go through the exact-order fallback."""
    qs = [query.random_graph(10 + seed, 7000 + seed, extra_edge_p=0.0, equal=True),
          query.random_graph(12 + seed, 7100 + seed, extra_edge_p=0.0),
          query.random_graph(13, 7200 + seed, extra_edge_p=0.0, rich=True),
          query.star(8 + seed, 7300 + seed, rich=True),
          query.chain(10 + seed, 7400 + seed)]
    for q in qs:
        want, _ = harness.run_port(q, 5)
        got = gpu_run(q, 5)
        assert same_tree(got.tree, want), q.name


def test_overflow_path_large_sets():
    """Sets with more candidates than one warp's share take the chunked
    atomicMin path (clique levels >= 12 in DPsub); compare with the oracle."""
    q = query.clique(13, 77)
    want, _ = harness.run_port(q, 3)
    got = gpu_run(q, 3)
    assert same_tree(got.tree, want)
    want5, _ = harness.run_port(q, 5)
    got5 = gpu_run(q, 5)
    assert same_tree(got5.tree, want5)


def _check_tree_arithmetic(q, tree):
    """Every internal node equals the oracle's join of its children."""
    n_nodes = 0

    def walk(t):
        nonlocal n_nodes
        n_nodes += 1
        if t[5] is None:
            assert t[6] is None
            return
        l, r = t[5], t[6]
        walk(l)
        walk(r)
        assert l[0] & r[0] == 0 and (l[0] | r[0]) == t[0]
        vals = harness.eval_join(q, l[0], r[0], l[1:5], r[1:5])
        assert (t[1], t[2], t[3], float(t[4])) == vals, (t[0], vals, t[1:5])

    walk(tree)
    assert n_nodes == 2 * q.n - 1
    full = 0
    for i in range(q.n):
        full |= 1 << (i + 1)
    assert tree[0] == full


@pytest.mark.parametrize("shape,n,seed", [("clique", 18, 0), ("snowflake", 28, 1), ("star", 20, 2)])
def test_full_size_properties(shape, n, seed):
    q = query.make(shape, n, seed)
    r5 = gpu_run(q, 5)
    _check_tree_arithmetic(q, r5.tree)
    again = gpu_run(q, 5)
    assert same_tree(r5.tree, again.tree)          # deterministic
    if shape == "clique":
        r3 = gpu_run(q, 3)
        _check_tree_arithmetic(q, r3.tree)
        assert r3.tree[3] == r5.tree[3]             # same optimum, both enumerators


DPSUB_GOLD = [c for c in GOLDEN if c["algorithm"] == 3]


def _csg(flag):
    C = __import__("ctypes")
    C.c_bool.in_dll(lib.load(), "gpuqo_dpsub_csg_enable").value = bool(flag)


@pytest.mark.parametrize("case", DPSUB_GOLD, ids=[f'{c["tag"]}-{c["name"]}' for c in DPSUB_GOLD])
def test_dpsub_all_subsets_enumeration(case):
    """gpuqo_dpsub_csg_enable off: plain DPsub tests every subset of every set
    (the reference's all-subsets enumeration with CCC); on (the default): only
    the valid csg-cmp pairs, keyed by their DPsub index.  Both return the
    reference's plan and cost the same valid pairs."""
    try:
        _csg(False)
        a = gpu_run(case["query"], 3)
    finally:
        _csg(True)
    b = gpu_run(case["query"], 3)
    assert same_tree(a.tree, case["expected"])
    assert same_tree(b.tree, case["expected"])
    assert a.stats["evaluated_pairs"] == b.stats["evaluated_pairs"]


@pytest.mark.parametrize("seed", range(6))
def test_dpsub_csg_ties_and_dense_graphs(seed):
    """Cost ties (all-equal graphs) and dense random graphs, where the DPsub
    and MPDP enumeration orders pick different winners among equal costs:
    the CSG path keeps DPsub's winner (the oracle restatement of cpu_dpsub)."""
    qs = [query.random_graph(9 + seed, 7000 + seed, equal=True),
          query.random_graph(8 + seed, 7100 + seed, extra_edge_p=0.5, rich=True),
          query.cycle(10 + seed, 7200 + seed), query.multi_member_classes(7 + seed, 7300 + seed)]
    for q in qs:
        want, _ = harness.run_port(q, 3)
        assert same_tree(gpu_run(q, 3).tree, want), q.name
