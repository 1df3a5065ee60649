"""Host-side multi-device dispatch (CPU): the split of a batch over devices
(gpuqo_b200_plan_shards, a pure host function of the library) and its
properties.  The library calls it with each query's estimated work and runs
every device's share on that device's own engines; with no data crossing
between devices, the split decides only the balance, never a plan."""
import ctypes as C
import random

import pytest

from gpuqo_b200 import lib


def _plan(work, n_dev):
    L = lib.load()
    f = L.gpuqo_b200_plan_shards
    f.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_int)]
    f.restype = C.c_int
    w = (C.c_double * len(work))(*work)
    out = (C.c_int * max(len(work), 1))()
    rc = f(w, len(work), n_dev, out)
    return rc, list(out)[:len(work)]


@pytest.mark.parametrize("n_dev", [1, 2, 3, 8])
@pytest.mark.parametrize("seed", range(5))
def test_split_is_balanced_and_deterministic(n_dev, seed):
    rng = random.Random(seed)
    # the batch mix's spread: a few huge items among many small ones
    work = [rng.choice([1.0, 10.0, 1e3, 1e6]) * rng.uniform(1, 2) for _ in range(200 + seed)]
    rc, dev = _plan(work, n_dev)
    assert rc == 0
    assert all(0 <= d < n_dev for d in dev)
    assert (rc, dev) == _plan(work, n_dev)                     # deterministic
    loads = [0.0] * n_dev
    for w, d in zip(work, dev):
        loads[d] += w
    # longest-processing-time bound: no device exceeds the least loaded one
    # by more than the largest item
    assert max(loads) - min(loads) <= max(work) + 1e-9
    if n_dev == 1:
        assert set(dev) == {0}


def test_split_orders_by_weight_then_index():
    rc, dev = _plan([5.0, 5.0, 5.0, 1.0], 2)
    assert rc == 0 and dev == [0, 1, 0, 1]
    rc, dev = _plan([], 4)
    assert rc == 0 and dev == []
    rc, _ = _plan([1.0], 0)
    assert rc == 1                                             # GPUQO_B200_ERR_ARGS
