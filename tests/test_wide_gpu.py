"""GPU parity of the sparse exact DP (the memo over connected sets only).

Exact DPsub and MPDP beyond 31 relations (the end of the dense memo) run on
the sparse memo: the connected sets are enumerated on the host, a device
open-addressing table maps each to its memo slot, and one launch per level
evaluates every set with 64-bit relation sets.  Checks:

* forced onto the sparse memo (gpuqo_b200_sparse_from_rels = 2), every golden
  case of up to 30 relations returns the reference's plan bit for bit, in
  both tie orders (DPsub and MPDP);
* at 32 to 63 relations the plan equals the oracle's (its sparse driver) bit
  for bit, and the root's total cost equals the optimum that the reference's
  cpu_dpccp reaches on the same query, its rows within 1e-6
  (wide_cases.jsonl: the reference's only exact DP that finishes at these
  sizes);
* the sparse memo serves IDP sub-problems and the planner service;
* limits end in a status, not a fault: too many connected sets
  (GPUQO_B200_ERR_TOO_LARGE, or GPUQO_B200_ERR_NOMEM under a device-memory
  budget), too many candidate splits (a large block that is not a cycle),
  DPsize beyond 31 relations (GPUQO_B200_ERR_UNSUPPORTED).
"""
import ctypes as C

import pytest

from conftest import load_golden, same_tree

import harness
from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu

ERR_NOMEM, ERR_TOO_LARGE, ERR_UNSUPPORTED = 3, 4, 5

SMALL = [c for c in load_golden() if c["query"].n <= 30]
WIDE = load_golden("wide_cases.jsonl")


@pytest.fixture
def knob():
    L = lib.load()
    yield lambda name, v: capi.set_int(L, name, v)
    capi.set_int(L, "gpuqo_b200_sparse_from_rels", 32)
    capi.set_int(L, "gpuqo_b200_device_memory_mb", 0)
    capi.set_int(L, "gpuqo_b200_sparse_host_list", 0)


def _run(q, alg, **kw):
    return lib.run(q, capi.GPUQO_DPSUB, bicc=(alg == 5), **kw)


@pytest.mark.parametrize("case", SMALL, ids=[f'{c["tag"]}-{c["name"]}-a{c["algorithm"]}' for c in SMALL])
def test_sparse_memo_returns_golden_plans(case, knob):
    knob("gpuqo_b200_sparse_from_rels", 2)
    r = _run(case["query"], case["algorithm"])
    assert r.error == 0, r.error
    assert same_tree(r.tree, case["expected"])


# cases whose oracle run takes minutes (DPsub lists every connected subset of
# every set; the 34-relation snowflake has 2.4 M sets): checked against the
# reference's optimum and the oracle's join arithmetic instead
NO_ORACLE = {("wide_snowflake32", 3), ("wide_snowflake34", 3), ("wide_snowflake34", 5)}


@pytest.mark.parametrize("alg", [3, 5])
@pytest.mark.parametrize("case", WIDE, ids=[c["tag"] for c in WIDE])
def test_wide_matches_oracle_and_reference_optimum(case, alg):
    q = case["query"]
    assert 32 <= q.n <= 63
    r = _run(q, alg)
    assert r.error == 0, r.error
    if (case["tag"], alg) in NO_ORACLE:
        _check_arithmetic(q, r.tree)
    else:
        want, _ = harness.run_port(q, alg)
        assert same_tree(r.tree, want), (q.name, alg)
    # the optimum: the root's total cost equal to DPccp's; its rows within
    # 1e-6 (a plan of equal cost in another tie order may multiply the same
    # selectivities in another order)
    ref = case["expected"]
    assert r.tree[3] == ref[3], (q.name, alg, r.tree[1:4], ref[1:4])
    assert abs(r.tree[1] - ref[1]) <= 1e-6 * abs(ref[1]), (q.name, alg, r.tree[1:4], ref[1:4])
    again = _run(q, alg)
    assert same_tree(again.tree, r.tree)       # deterministic, and the scratch is reusable


def test_wide_serves_idp_subproblems_and_the_service():
    """IDP2 with 40-relation sub-problems on a 60-relation chain of key joins:
    every sub-problem above 31 relations runs on the sparse memo; the plan
    covers the relations and each join is the oracle's arithmetic of its
    children (the oracle takes at most 63 relations).  The same request
    through the service returns the same plan."""
    q = query.key_chain(60, 21)
    r = lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=40, idp_type=capi.GPUQO_IDP2)
    assert r.error == 0
    _check_arithmetic(q, r.tree)
    srv = lib.Server(max_inflight=4, wave_memory_mb=1024)
    try:
        t = srv.submit(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=40, idp_type=capi.GPUQO_IDP2)
        wide = query.key_cycle(44, 22)
        t2 = srv.submit(wide, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=0, idp_type=capi.GPUQO_IDP2)
        rc, tree, _ = srv.wait(t)
        rc2, tree2, _ = srv.wait(t2)
    finally:
        srv.stop()
    assert rc == 0 and same_tree(tree, r.tree)
    assert rc2 == 0 and same_tree(tree2, harness.run_port(wide, 5)[0])


def _check_arithmetic(q, tree):
    n_nodes = 0

    def walk(t):
        nonlocal n_nodes
        n_nodes += 1
        if t[5] is None:
            return
        l, r = t[5], t[6]
        walk(l)
        walk(r)
        assert l[0] & r[0] == 0 and (l[0] | r[0]) == t[0]
        assert (t[1], t[2], t[3], float(t[4])) == harness.eval_join(q, l[0], r[0], l[1:5], r[1:5])

    walk(tree)
    assert n_nodes == 2 * q.n - 1


def _ladder(n_rungs, seed):
    """Two chains of key joins joined rung by rung: one biconnected block of
    every relation that is not a cycle."""
    import numpy as np
    from gpuqo_b200.query import _assemble, _key_edges, _loguniform
    n = 2 * n_rungs
    rng = np.random.default_rng([seed, 14, n])
    lrows = _loguniform(rng, 1e2, 1e7, n)
    pairs = ([(i, i + 1) for i in range(n_rungs - 1)] + [(n_rungs + i, n_rungs + i + 1) for i in range(n_rungs - 1)] +
             [(i, n_rungs + i) for i in range(n_rungs)])
    return _assemble(f"ladder{n}_s{seed}", n, lrows, [8] * n, _key_edges(pairs, lrows), rng)


def _equalized(q, rows):
    """The same graph with identical relations and identical plain classes:
    most splits of a set cost exactly the same, so the plan is decided by the
    tie order alone.  With 100 rows and selectivity 0.01 every join keeps 100
    rows; with 1000 the estimates overflow to inf and the costs to inf and
    NaN (the reference's NaN rule decides)."""
    from gpuqo_b200.query import EqClass, VarInfo
    q.rows = [float(rows)] * q.n
    q.tuples = [float(rows)] * q.n
    q.startup = [0.0] * q.n
    q.total = [18.0] * q.n
    q.width = [8] * q.n
    q.eq_classes = [EqClass(list(e.members), [0.01] * len(e.sels), [[] for _ in e.members],
                            [VarInfo() for _ in e.members]) for e in q.eq_classes]
    q.name = f"equal{rows}_" + q.name
    return q


@pytest.mark.parametrize("rows", [100, 1000])
@pytest.mark.parametrize("alg", [3, 5])
@pytest.mark.parametrize("make", [lambda: query.key_chain(40, 31), lambda: query.key_cycle(36, 32),
                                  lambda: query.lollipop(42, 33), lambda: query.ring_path(38, 34)],
                         ids=["chain40", "cycle36", "lollipop42", "ring_path38"])
def test_wide_ties_follow_the_reference_order(make, alg, rows):
    """32 to 63 relations where nearly every split ties: tree path (chain),
    cycle arcs, blocks joined by bridges; the oracle's plan bit for bit."""
    q = _equalized(make(), rows)
    r = _run(q, alg)
    assert r.error == 0, r.error
    want, _ = harness.run_port(q, alg)
    assert same_tree(r.tree, want), (q.name, alg)


@pytest.mark.parametrize("alg", [3, 5])
@pytest.mark.parametrize("case", [c for c in WIDE if c["tag"] in ("wide_key_cycle48_rich", "wide_lollipop63_rich",
                                                                     "wide_ring_path40", "wide_ring_path36_rich")],
                         ids=lambda c: c["tag"])
def test_device_listing_of_general_graphs(case, alg, knob):
    """Graphs with cycles list their connected sets on the host up to
    gpuqo_b200_sparse_host_list sets and on the device beyond; with the limit
    at 1 every level is listed on the device: the oracle's plan bit for bit."""
    q = case["query"]
    knob("gpuqo_b200_sparse_host_list", 1)
    r = _run(q, alg)
    assert r.error == 0, r.error
    assert r.stats["connected_sets"] == len_connected_sets(q) - q.n
    want, _ = harness.run_port(q, alg)
    assert same_tree(r.tree, want), (q.name, alg)


def len_connected_sets(q):
    adj = [0] * q.n
    for i, e in enumerate(q.edges):
        for j in e:
            adj[i] |= 1 << j
    cur = {1 << i for i in range(q.n)}
    total = len(cur)
    while cur:
        nxt = set()
        for S in cur:
            N, x = 0, S
            while x:
                N |= adj[(x & -x).bit_length() - 1]
                x &= x - 1
            N &= ~S
            while N:
                nxt.add(S | (N & -N))
                N &= N - 1
        total += len(nxt)
        cur = nxt
    return total


def test_tree_path_matches_dense_memo(knob):
    """Tree-shaped graphs take the sparse memo's tree path (sets listed on the
    device, edge-wise candidates from per-root tables, no block search): on a
    28-relation snowflake (dense memo of 5.4 GB) and a 24-relation star its plans
    equal the dense engine's bit for bit, for MPDP and plain DPsub."""
    for q in (query.snowflake(28, 1), query.star(24, 3), query.snowflake(26, 9, rich=True)):
        for alg in (3, 5):
            dense = _run(q, alg)
            knob("gpuqo_b200_sparse_from_rels", 2)
            sparse = _run(q, alg)
            knob("gpuqo_b200_sparse_from_rels", 32)
            assert dense.error == 0 and sparse.error == 0
            assert same_tree(sparse.tree, dense.tree), (q.name, alg)


def test_wide_limits_end_in_a_status(knob):
    # a star of 34: 2^33 connected sets
    r = _run(query.star(34, 23), 5)
    assert r.tree is None and r.error == ERR_TOO_LARGE
    # the same under a budget of 64 MB: refused as out of memory, early
    knob("gpuqo_b200_device_memory_mb", 64)
    r = _run(query.star(34, 23), 5)
    assert r.tree is None and r.error == ERR_NOMEM
    knob("gpuqo_b200_device_memory_mb", 0)
    # a 32-relation ladder: few connected sets, but blocks of up to 32
    # relations that are not cycles (2^32 splits for the whole set)
    r = _run(_ladder(16, 24), 5)
    assert r.tree is None and r.error == ERR_TOO_LARGE
    # DPsize has no sparse memo
    r = lib.run(query.key_chain(40, 25), capi.GPUQO_DPSIZE)
    assert r.tree is None and r.error == ERR_UNSUPPORTED
    # and the library is unaffected
    q = WIDE[0]["query"]
    assert same_tree(_run(q, 5).tree, harness.run_port(q, 5)[0])
