"""GPU test of the autotuner (gpuqo_b200_autotune): it measures the kernel
variant and batch hand-off crossovers on the device and installs them; plans
are the same before and after, for single queries across the size range and
for a batch."""
import pytest

from conftest import same_tree

from gpuqo_b200 import capi, lib, query

pytestmark = pytest.mark.gpu


def _plans():
    qs = [query.star(n, 300 + n) for n in (15, 19, 21, 23)] + [query.snowflake(25, 301), query.chain(28, 302)]
    single = [lib.run(q, capi.GPUQO_DPSUB, bicc=True).tree for q in qs]
    batch, rc = lib.run_batch(qs + query.batch_mix(40, seed=303, nmin=8, nmax=16), capi.GPUQO_DPSUB, bicc=True)
    assert rc == 0
    return single, batch


def test_autotune_installs_crossovers_without_changing_plans():
    before = _plans()
    try:
        t = lib.autotune()
        assert t["tuned"] == 1 and t["tune_ms"] > 0.0
        for k in ("single_narrow_level_sets", "single_wide_level_sets", "batch_single_sets"):
            assert t[k] >= 0.0
        assert lib.get_tuning() == t
        after = _plans()
        for a, b in zip(before[0] + before[1], after[0] + after[1]):
            assert same_tree(a, b)
    finally:
        # the built-in crossovers again, for the tests after this one
        lib.set_tuning(16384.0, 1e30, float(1 << 20), tuned=0)
