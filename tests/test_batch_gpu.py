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


def test_batch_persistent_matches_level_launches():
    """One cooperative launch per wave (kb_dp) and the per-level launches
    return the same plans, counters and pair counts."""
    # n <= 11 keeps every cycle inside the batched kernel's candidate bound
    qs = query.batch_mix(240, seed=5, nmin=2, nmax=11)
    l = lib.load()
    out = {}
    try:
        for p in (1, 0):
            capi.set_int(l, "gpuqo_b200_persistent", p)
            trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
            assert rc == 0
            out[p] = (trees, lib.get_stats())
    finally:
        capi.set_int(l, "gpuqo_b200_persistent", 1)
    (tp, sp), (tl, sl) = out[1], out[0]
    for q, a, b in zip(qs, tp, tl):
        assert same_tree(a, b), q.name
    assert sp["n_subproblems"] == len(qs)
    assert sp["kernel_launches"] == 2          # one wave of tree-shaped queries, one of cycles
    assert sl["kernel_launches"] > 2 * 9
    assert sp["connected_sets"] == sl["connected_sets"]
    assert sp["evaluated_pairs"] == sl["evaluated_pairs"]


@pytest.mark.parametrize("persistent", [1, 0])
def test_batch_large_blocks(persistent):
    """Sets with more candidates than one group evaluates (the full set of a
    cycle of 12+ relations, dense random graphs) take kb_dp's overflow phase;
    without the persistent kernel those queries run on the single engine.
    Either way every plan equals gpuqo_run's and the oracle's."""
    qs = ([query.cycle(n, 60 + n) for n in (12, 13, 15, 18, 21)] +
          [query.random_graph(n, 70 + n, extra_edge_p=0.45, rich=True) for n in (12, 14, 15)] +
          [query.star(n, 80 + n) for n in (9, 14)] + [query.snowflake(16, 91)])
    l = lib.load()
    try:
        capi.set_int(l, "gpuqo_b200_persistent", persistent)
        trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    finally:
        capi.set_int(l, "gpuqo_b200_persistent", 1)
    assert rc == 0
    for q, t in zip(qs, trees):
        single = lib.run(q, capi.GPUQO_DPSUB, bicc=True)
        assert same_tree(t, single.tree), q.name
        if q.n <= 15:
            want, _ = harness.run_port(q, 5)
            assert same_tree(t, want), q.name


def test_batch_large_tree_runs_alone():
    """A tree-shaped query with more connected sets than the hand-off
    threshold (2^20 by default, or what the autotuner measured; a 22-relation
    star has 2^21 + 21) leaves the wave for the single-query kernel; the
    plans are those of gpuqo_run."""
    qs = [query.star(22, 123)] + [query.star(10, 130 + i) for i in range(3)] + [query.snowflake(14, 140)]
    trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    alone = (1 << 21) + 21 > lib.get_tuning()["batch_single_sets"]
    # k_dp_tree for the star when it runs alone, kb_dp for the wave
    assert lib.get_stats()["kernel_launches"] == (2 if alone else 1)
    for q, t in zip(qs, trees):
        assert same_tree(t, lib.run(q, capi.GPUQO_DPSUB, bicc=True).tree), q.name


def test_batch_plain_dpsub_rides_the_batch():
    """Plain DPsub (bicc off) with gpuqo_dpsub_csg_enable runs in the batched
    kernel as well; every plan is cpu_dpsub's."""
    qs = query.batch_mix(48, seed=8, nmin=6, nmax=13)   # sparse: below half of all possible edges
    trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=False)
    assert rc == 0
    assert lib.get_stats()["kernel_launches"] == 2   # tree-shaped queries, then cycles
    for q, t in zip(qs, trees):
        want, _ = harness.run_port(q, 3)
        assert same_tree(t, want), q.name


def test_batch_mix_8_28_sample_vs_oracle():
    """A sample of the benchmark's own batched workload (4096 queries, shapes
    40/40/10/10, relation counts uniform in [8, 28], seed 7): every 50th query
    of at most 22 relations (stars of at most 19, whose oracle run grows as
    2^n), batched together, against the oracle restatement of cpu_dpsub_bicc."""
    qs = query.batch_mix(4096, seed=7, nmin=8, nmax=28)
    eligible = [q for q in qs if q.n <= 22 and not (q.name.startswith("star") and q.n > 19)]
    sample = eligible[::50]
    assert len(sample) >= 40
    trees, rc = lib.run_batch(sample, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    for q, t in zip(sample, trees):
        want, _ = harness.run_port(q, 5)
        assert same_tree(t, want), q.name
