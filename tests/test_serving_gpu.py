"""GPU tests of the continuous-batching planner service: every request's plan
equals the plan gpuqo_run returns for the same query alone, whether it runs
alone or overlapped with other requests (IDP2, UnionDP and exact DPs mixed),
and the service reports its waves."""
import threading

import pytest

from conftest import same_tree

from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu


def _workload():
    reqs = []
    for i in range(6):
        reqs.append((query.snowflake(30 + 9 * i, 1200 + i), 10 + i, capi.GPUQO_IDP2))
    for i in range(4):
        reqs.append((query.snowflake(32 + 7 * i, 1300 + i, rich=True), 12, capi.GPUQO_UNION))
    for i in range(8):
        reqs.append((query.batch_mix(1, 1400 + i, 6, 14)[0], 0, capi.GPUQO_IDP2))
    return reqs


def test_serving_same_plan_alone_and_in_mix():
    reqs = _workload()
    alone = [lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t).tree for (q, k, t) in reqs]
    srv = lib.Server(max_inflight=8, wave_memory_mb=4096)
    try:
        # one at a time through the service
        for (q, k, t), want in zip(reqs, alone):
            tk = srv.submit(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t)
            rc, got, lat = srv.wait(tk)
            assert rc == 0 and same_tree(got, want), q.name
        # all at once, waited for from several threads
        tickets = [srv.submit(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t) for (q, k, t) in reqs]
        results = [None] * len(tickets)

        def waiter(j):
            results[j] = srv.wait(tickets[j])

        ths = [threading.Thread(target=waiter, args=(j,)) for j in range(len(tickets))]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        for (rc, got, lat), want, (q, _, _) in zip(results, alone, reqs):
            assert rc == 0 and same_tree(got, want), q.name
            assert lat > 0
        st = srv.stats()
        assert st["completed"] == 2 * len(reqs)
        assert st["waves"] >= 1 and st["batched_subproblems"] >= len(reqs)
    finally:
        srv.stop()
