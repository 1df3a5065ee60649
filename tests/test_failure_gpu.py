"""GPU: failure paths, injected on the host (no device fault is ever caused).

* a device-memory budget below a query's need: GPUQO_B200_ERR_NOMEM before
  anything is allocated, and the next call that fits returns the reference's
  plan (single query, batch);
* a disconnected query graph: GPUQO_B200_ERR_ARGS from gpuqo_run;
* a served mix in which one request has a disconnected graph and another is
  cancelled in the middle of its IDP iterations: those two report their
  status, every other request returns the plan it returns alone.

The grid-barrier timeout of the persistent kernels is exercised in
test_persistent_gpu.py (gpuqo_b200_barrier_poll_limit).
"""
import threading

import pytest

from conftest import same_tree

import harness
from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu

ERR_ARGS, ERR_NOMEM, ERR_CANCELLED = 1, 3, 6


def _disconnected(n, seed):
    """A chain with its middle edge (and that edge's class) removed."""
    q = query.chain(n, seed)
    a = next(i for i in range(n) if len(q.edges[i]) == 1)   # one end of the chain
    # walk to the middle edge
    prev, cur = -1, a
    for _ in range(n // 2 - 1):
        nxt = next(j for j in q.edges[cur] if j != prev)
        prev, cur = cur, nxt
    mid = next(j for j in q.edges[cur] if j != prev)
    q.edges[cur] = [j for j in q.edges[cur] if j != mid]
    q.edges[mid] = [j for j in q.edges[mid] if j != cur]
    q.eq_classes = [e for e in q.eq_classes if sorted(e.members) != sorted([cur, mid])]
    q.name = f"disconnected{n}_s{seed}"
    return q


@pytest.fixture
def budget():
    L = lib.load()
    yield lambda mb: capi.set_int(L, "gpuqo_b200_device_memory_mb", mb)
    capi.set_int(L, "gpuqo_b200_device_memory_mb", 0)


def test_memory_budget_refuses_then_next_call_succeeds(budget):
    q = query.snowflake(21, 41)                 # dense memo 2^21 x 20 B = 42 MB
    want, _ = harness.run_port(q, 5)
    budget(16)
    r = lib.run(q, capi.GPUQO_DPSUB, bicc=True)
    assert r.tree is None and r.error == ERR_NOMEM
    small = query.snowflake(12, 42)             # fits the budget
    assert same_tree(lib.run(small, capi.GPUQO_DPSUB, bicc=True).tree, harness.run_port(small, 5)[0])
    budget(0)
    r = lib.run(q, capi.GPUQO_DPSUB, bicc=True)
    assert r.error == 0 and same_tree(r.tree, want)


def test_memory_budget_batch(budget):
    qs = [query.cycle(19, 43), query.snowflake(10, 44)]
    want = [harness.run_port(q, 5)[0] for q in qs]
    budget(8)
    trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == ERR_NOMEM
    budget(0)
    trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0 and all(same_tree(a, b) for a, b in zip(trees, want))


def test_disconnected_graph_is_refused():
    q = _disconnected(12, 45)
    for bicc in (True, False):
        r = lib.run(q, capi.GPUQO_DPSUB, bicc=bicc)
        assert r.tree is None and r.error == ERR_ARGS


def test_served_mix_with_failing_and_cancelled_requests():
    ok_reqs = ([(query.snowflake(40 + 11 * i, 1500 + i), 12, capi.GPUQO_IDP2) for i in range(4)] +
               [(query.snowflake(35 + 5 * i, 1510 + i, rich=True), 12, capi.GPUQO_UNION) for i in range(3)] +
               [(query.batch_mix(1, 1520 + i, 8, 16)[0], 0, capi.GPUQO_IDP2) for i in range(5)])
    alone = [lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t).tree for (q, k, t) in ok_reqs]
    bad = _disconnected(40, 1530)
    # a long IDP2 request (about 60 sub-problems), cancelled right after it
    # is submitted: the cancel reaches it before one of its exact DPs
    doomed = query.snowflake(900, 1531)
    srv = lib.Server(max_inflight=8, wave_memory_mb=4096)
    try:
        t_doomed = srv.submit(doomed, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=16, idp_type=capi.GPUQO_IDP2)
        assert srv.cancel(t_doomed) == 0
        tickets = [srv.submit(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t) for (q, k, t) in ok_reqs]
        t_bad = srv.submit(bad, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=12, idp_type=capi.GPUQO_IDP2)
        results = [None] * len(tickets)

        def waiter(j):
            results[j] = srv.wait(tickets[j])

        ths = [threading.Thread(target=waiter, args=(j,)) for j in range(len(tickets))]
        for th in ths:
            th.start()
        rc_doomed, tree_doomed, _ = srv.wait(t_doomed)
        rc_bad, tree_bad, _ = srv.wait(t_bad)
        for th in ths:
            th.join()
        assert rc_doomed == ERR_CANCELLED and tree_doomed is None
        assert rc_bad == ERR_ARGS and tree_bad is None
        for (rc, got, _), want, (q, _, _) in zip(results, alone, ok_reqs):
            assert rc == 0 and same_tree(got, want), q.name
        assert srv.cancel(t_doomed) == ERR_ARGS      # already waited for: unknown ticket
    finally:
        srv.stop()
