"""CPU tests of the C ABI: the product library loads, exports every symbol
include/gpuqo_b200.h declares, and the ctypes mirror of the reference structs
has the reference's layout.  No compute call is made (no GPU here)."""
import ctypes as C
import math

import pytest

from gpuqo_b200 import capi, lib


def test_library_exports_declared_symbols():
    l = lib.load()
    syms = lib.declared_symbols()
    assert "gpuqo_run" in syms and "gpuqo_dpsub_bicc_enable" in syms
    missing = [s for s in syms if not hasattr(l, s)]
    assert not missing, missing


def test_guc_boot_values():
    """The values the library's GUC variables hold as it is loaded (recorded
    by lib.load(), so that tests run before this one in the same process and
    changing them do not matter): the boot values of
    src/backend/utils/misc/guc.c."""
    lib.load()
    b = lib.boot_gucs
    assert b["gpuqo_n_parallel"] == 10240
    assert b["gpuqo_dpsub_filter_threshold"] == 16
    assert b["gpuqo_idp_type"] == capi.GPUQO_IDP2
    assert b["gpuqo_idp_n_iters"] == 0
    assert b["gpuqo_dpsub_ccc_enable"] is True
    assert b["gpuqo_dpsub_bicc_enable"] is False
    assert b["gpuqo_dpsub_csg_enable"] is True


def test_struct_layouts_match_reference():
    # LP64 layouts of src/include/optimizer/gpuqo_planner_info.h / gpuqo_common.h
    assert C.sizeof(capi.PathCost) == 8
    assert C.sizeof(capi.GpuqoIndexInfo) == 16
    assert C.sizeof(capi.VarInfoC) == 28
    assert C.sizeof(capi.BaseRelationC) == 32
    assert C.sizeof(capi.EqClassInfo) == 48
    assert C.sizeof(capi.GpuqoPlannerInfoC) == 48
    assert C.sizeof(capi.QueryTreeC) == 40
    assert capi.GpuqoPlannerInfoC.n_eq_classes.offset == 32


def test_bitmapset_roundtrip():
    for bits in (0b10, 1 << 63, (1 << 64) | 2, (1 << 200) | (1 << 65) | 4):
        b = capi.make_bitmapset(bits)
        assert capi.read_bitmapset(C.addressof(b)) == bits


def test_cancel_request_returns_null_before_any_device_work():
    """With InterruptPending set (Postgres's cancel flag, a weak symbol that the
    backend's own definition replaces), gpuqo_run returns NULL with
    GPUQO_B200_ERR_CANCELLED before touching the GPU, so it runs here."""
    from gpuqo_b200 import query
    l = lib.load()
    flag = C.c_int.in_dll(l, "InterruptPending")
    b = capi.PlannerInfoBuilder(query.star(6, 1))
    try:
        flag.value = 1
        for idp in (0, 3):   # exact DP, and the IDP driver
            capi.set_int(l, "gpuqo_idp_n_iters", idp)
            assert not l.gpuqo_run(capi.GPUQO_DPSUB, b.pointer())
            assert l.gpuqo_b200_last_error() == 6   # GPUQO_B200_ERR_CANCELLED
    finally:
        flag.value = 0
        capi.set_int(l, "gpuqo_idp_n_iters", 0)


def test_tuning_defaults_before_autotune():
    """Until gpuqo_b200_autotune runs, the built-in choices apply: the
    2-blocks-per-SM tree kernel up to 16384 connected sets per relation and
    the 3-blocks-per-SM one above, batches hand tree queries of more than
    2^20 connected sets to single launches."""
    t = lib.get_tuning()
    assert t["tuned"] == 0 and t["tune_ms"] == 0.0
    assert t["single_narrow_level_sets"] == 16384.0
    assert t["single_wide_level_sets"] >= 1e29
    assert t["batch_single_sets"] == float(1 << 20)


def test_set_tuning_installs_and_rejects():
    """gpuqo_b200_set_tuning installs saved crossovers without measuring
    (get_tuning reads them back), rejects negative and NaN ones, and restoring
    the defaults with tuned = 0 gives back the untuned state."""
    lib.set_tuning(5000.0, 80000.0, 123456.0)
    t = lib.get_tuning()
    assert (t["single_narrow_level_sets"], t["single_wide_level_sets"], t["batch_single_sets"], t["tuned"]) == \
        (5000.0, 80000.0, 123456.0, 1)
    for bad in ((-1.0, 1.0, 1.0), (1.0, math.nan, 1.0), (1.0, 1.0, -2.0)):
        with pytest.raises(ValueError):
            lib.set_tuning(*bad)
    assert lib.get_tuning() == t
    lib.set_tuning(16384.0, 1e30, float(1 << 20), tuned=0)
    t = lib.get_tuning()
    assert t["tuned"] == 0 and t["tune_ms"] == 0.0 and t["single_narrow_level_sets"] == 16384.0

