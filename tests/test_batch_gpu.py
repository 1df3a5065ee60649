"""GPU tests of the batched entry point gpuqo_b200_run_batch: every plan of a
batch equals the plan gpuqo_run returns for the same query alone, and the
oracle's, for the batched workload's shape mix (star / snowflake / chain /
cycle) at sizes the oracle runs quickly; waves (memory budget) and mixed
algorithms do not change any plan."""
import pytest

from conftest import same_tree

import harness
from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu


def test_batch_matches_single_and_oracle():
    qs = query.batch_mix(160, seed=3, nmin=3, nmax=14)
    trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    st = lib.get_stats()
    assert st["n_subproblems"] == len(qs)
    for q, t in zip(qs, trees):
        single = lib.run(q, capi.GPUQO_DPSUB, bicc=True)
        assert same_tree(t, single.tree), q.name
        want, _ = harness.run_port(q, 5)
        assert same_tree(t, want), q.name


def test_batch_waves_do_not_change_plans():
    qs = query.batch_mix(60, seed=4, nmin=8, nmax=18)
    ref, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    l = lib.load()
    import ctypes as C
    old = C.c_int.in_dll(l, "gpuqo_b200_batch_memory_mb").value
    try:
        C.c_int.in_dll(l, "gpuqo_b200_batch_memory_mb").value = 64   # many small waves
        waves, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    finally:
        C.c_int.in_dll(l, "gpuqo_b200_batch_memory_mb").value = old
    assert rc == 0
    for a, b in zip(ref, waves):
        assert same_tree(a, b)


def test_batch_plain_dpsub_and_general_graphs():
    qs = [query.random_graph(9, 40 + i, extra_edge_p=0.3, rich=True) for i in range(6)] + \
         [query.star(9, 50 + i) for i in range(4)]
    for alg, bicc in ((capi.GPUQO_DPSUB, False), (capi.GPUQO_DPSUB, True)):
        trees, rc = lib.run_batch(qs, alg, bicc=bicc)
        assert rc == 0
        for q, t in zip(qs, trees):
            want, _ = harness.run_port(q, 5 if bicc else 3)
            assert same_tree(t, want), (q.name, bicc)
