"""GPU: the multi-device paths of the batch entry and the planner service
(gpuqo_b200_devices).  On a box with one GPU, gpuqo_b200_devices = 2 maps both
shards (both service lanes) to that GPU, so the split, the per-device host
threads and the merge of their results run for real; every plan must equal
the plan of the one-device path, bit for bit."""
import pytest

from conftest import same_tree

from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu


@pytest.fixture
def two_devices():
    L = lib.load()
    capi.set_int(L, "gpuqo_b200_devices", 2)
    yield
    capi.set_int(L, "gpuqo_b200_devices", 1)


def test_batch_split_over_two_devices(two_devices):
    qs = query.batch_mix(96, seed=31, nmin=8, nmax=18)
    L = lib.load()
    capi.set_int(L, "gpuqo_b200_devices", 1)
    want, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    capi.set_int(L, "gpuqo_b200_devices", 2)
    got, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    assert all(same_tree(a, b) for a, b in zip(got, want))


def test_service_with_two_lanes(two_devices):
    reqs = ([(query.snowflake(30 + 7 * i, 1600 + i), 12, capi.GPUQO_IDP2) for i in range(4)] +
            [(query.batch_mix(1, 1610 + i, 8, 16)[0], 0, capi.GPUQO_IDP2) for i in range(6)])
    alone = [lib.run(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t).tree for (q, k, t) in reqs]
    srv = lib.Server(max_inflight=8, wave_memory_mb=4096)
    try:
        tickets = [srv.submit(q, capi.GPUQO_DPSUB, bicc=True, idp_n_iters=k, idp_type=t) for (q, k, t) in reqs]
        for tk, want, (q, _, _) in zip(tickets, alone, reqs):
            rc, got, _ = srv.wait(tk)
            assert rc == 0 and same_tree(got, want), q.name
    finally:
        srv.stop()
