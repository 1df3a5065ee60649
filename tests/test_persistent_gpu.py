"""GPU: the persistent tree-mode MPDP kernel (one cooperative launch per DP,
grid barrier between levels) against the per-level launches and the oracle.

gpuqo_b200_persistent selects the path (default 1).  Both paths must return
bit-identical plans; the persistent one must report a single kernel launch,
and queries that are not tree-shaped must keep the per-level path.
"""
import ctypes as C

import pytest

from conftest import same_tree

import harness
from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu


def _run(q, persistent):
    capi.set_int(lib.load(), "gpuqo_b200_persistent", 1 if persistent else 0)
    try:
        r = lib.run(q, capi.GPUQO_DPSUB, bicc=True, ccc=True)
    finally:
        capi.set_int(lib.load(), "gpuqo_b200_persistent", 1)
    assert r.error == 0, f"gpuqo_b200 error {r.error}"
    return r


TREES = ([query.star(n, 100 + n) for n in (2, 3, 8, 13, 18)] +
         [query.snowflake(n, 200 + n, rich=(n % 2 == 0)) for n in (6, 11, 17, 22, 25)] +
         [query.chain(n, 300 + n) for n in (4, 9, 20, 30)] +
         [query.random_graph(n, 400 + n, extra_edge_p=0.0, rich=True) for n in (5, 12, 19, 24)] +
         [query.random_graph(n, 500 + n, extra_edge_p=0.0, equal=True) for n in (7, 14, 21)])


@pytest.mark.parametrize("q", TREES, ids=[q.name for q in TREES])
def test_persistent_matches_level_launches(q):
    a = _run(q, True)
    b = _run(q, False)
    assert same_tree(a.tree, b.tree)
    assert a.stats["kernel_launches"] == 1
    assert b.stats["kernel_launches"] > 1
    assert a.stats["connected_sets"] == b.stats["connected_sets"]
    assert a.stats["evaluated_pairs"] == b.stats["evaluated_pairs"]


@pytest.mark.parametrize("q", [t for t in TREES if t.n <= 20], ids=[t.name for t in TREES if t.n <= 20])
def test_persistent_vs_oracle(q):
    want, _ = harness.run_port(q, 5)
    assert same_tree(_run(q, True).tree, want)


def test_persistent_sizes_in_a_row():
    """Counters and the barrier words are reset per run:
    sizes up, down and repeated give the plans of fresh runs."""
    qs = [query.snowflake(n, 700 + n) for n in (9, 20, 9, 15, 20, 4)]
    want = {q.name: _run(q, False).tree for q in qs}
    for q in qs:
        assert same_tree(_run(q, True).tree, want[q.name])


NOT_TREES = [query.cycle(12, 801), query.cycle(22, 803), query.clique(7, 802),
             query.random_graph(14, 804, extra_edge_p=0.3, rich=True),
             # a class of three or more members joins every pair of them
             query.multi_member_classes(6, 606), query.multi_member_classes(12, 612)]


@pytest.mark.parametrize("q", NOT_TREES, ids=[q.name for q in NOT_TREES])
def test_not_tree_single_launch(q):
    """Graphs with cycles run as a one-query wave of the general persistent
    kernel (kb_dp, overflow phases in the same launch); with
    gpuqo_b200_persistent = 0 as per-level launches; both give the oracle's
    plan."""
    a = _run(q, True)
    b = _run(q, False)
    assert a.stats["kernel_launches"] == 1
    assert b.stats["kernel_launches"] > 1
    assert a.stats["evaluated_pairs"] == b.stats["evaluated_pairs"]
    want, _ = harness.run_port(q, 5)
    assert same_tree(a.tree, want)
    assert same_tree(b.tree, want)


@pytest.mark.parametrize("warmup,iters", [(0, 1), (2, 3)])
def test_time_resident_uses_persistent(warmup, iters):
    """The device-resident timer takes the same single-launch path, with or
    without warm-up replays, and returns the plan of gpuqo_run."""
    q = query.snowflake(16, 901)
    want = _run(q, False).tree
    rc, ms, tree, st = lib.time_resident(q, capi.GPUQO_DPSUB, bicc=True, warmup=warmup, iters=iters)
    assert rc == 0 and ms > 0.0
    assert st["kernel_launches"] == 1
    assert st["eval_kernel_launches"] == iters
    assert same_tree(tree, want)


# crossovers (connected sets per level) that pin one occupancy variant of the
# persistent tree kernel: 2, 3 or 4 blocks per SM
VARIANTS = {"2_blocks": (1e30, 1e30), "3_blocks": (0.0, 1e30), "4_blocks": (0.0, 0.0)}
_LEVEL_PLANS = {}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_each_variant_matches_level_launches(variant):
    """Pinned with gpuqo_b200_set_tuning, each occupancy variant of the
    persistent kernel (the 2- and 3-blocks ones with the software-pipelined
    candidate loop, the 4-blocks one with the plain loop) returns the plan of
    the per-level path on every tree, and the oracle's on the small ones."""
    narrow, wide = VARIANTS[variant]
    saved = lib.get_tuning()
    lib.set_tuning(narrow, wide, saved["batch_single_sets"], tuned=saved["tuned"])
    try:
        for q in TREES:
            if q.name not in _LEVEL_PLANS:
                _LEVEL_PLANS[q.name] = _run(q, False).tree
            a = _run(q, True)
            assert a.stats["kernel_launches"] == 1
            assert same_tree(a.tree, _LEVEL_PLANS[q.name]), q.name
            if q.n <= 14:
                want, _ = harness.run_port(q, 5)
                assert same_tree(a.tree, want), q.name
    finally:
        lib.set_tuning(saved["single_narrow_level_sets"], saved["single_wide_level_sets"],
                       saved["batch_single_sets"], tuned=saved["tuned"])



def _reset_latch():
    L = lib.load()
    L.gpuqo_b200_reset_persistent.restype = C.c_int
    return L.gpuqo_b200_reset_persistent()


def test_barrier_timeout_reruns_per_level_and_latches():
    """A grid-barrier wait that runs out (gpuqo_b200_barrier_poll_limit = 1:
    a block gives up after one poll unless every block has already arrived)
    raises the kernel's error flag; the host reruns the DP with per-level
    launches, returns the per-level plan, and keeps the engine on per-level
    launches until gpuqo_b200_reset_persistent()."""
    L = lib.load()
    q = query.snowflake(20, 3)
    want = _run(q, False).tree
    assert same_tree(want, harness.run_port(q, 5)[0])
    try:
        capi.set_int(L, "gpuqo_b200_barrier_poll_limit", 1)
        first = _run(q, True)
        assert first.stats["barrier_timeouts"] == 1
        assert same_tree(first.tree, want)
        # latched: no second persistent attempt, per-level launches straight away
        again = _run(q, True)
        assert again.stats["barrier_timeouts"] == 0
        assert again.stats["kernel_launches"] > 1
        assert same_tree(again.tree, want)
    finally:
        capi.set_int(L, "gpuqo_b200_barrier_poll_limit", 0)
    assert _reset_latch() >= 1
    back = _run(q, True)
    assert back.stats["kernel_launches"] == 1 and back.stats["barrier_timeouts"] == 0
    assert same_tree(back.tree, want)


def test_batch_wave_barrier_timeout_reruns_per_level():
    """The same for a batch wave (kb_dp): the timed-out wave is rerun with
    per-level launches and every plan equals gpuqo_run's."""
    L = lib.load()
    qs = [query.snowflake(n, 800 + n) for n in (8, 10, 12, 14)] + [query.cycle(n, 850 + n) for n in (7, 11)]
    want = [_run(q, False).tree for q in qs]
    try:
        capi.set_int(L, "gpuqo_b200_barrier_poll_limit", 1)
        trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
        assert rc == 0 and lib.get_stats()["barrier_timeouts"] >= 1
        assert all(same_tree(a, b) for a, b in zip(trees, want))
    finally:
        capi.set_int(L, "gpuqo_b200_barrier_poll_limit", 0)
    _reset_latch()
    trees, rc = lib.run_batch(qs, capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0 and lib.get_stats()["barrier_timeouts"] == 0
    assert all(same_tree(a, b) for a, b in zip(trees, want))
