import json
import math
import os
import struct
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "postgres-gpuqo_b200"), os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden", "cases.jsonl")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: minutes-long case")


def load_golden(name="cases.jsonl"):
    from gpuqo_b200.query import Query
    out = []
    with open(os.path.join(REPO, "tests", "golden", name)) as f:
        for line in f:
            rec = json.loads(line)
            rec["query"] = Query.from_dict(rec["query"])
            out.append(rec)
    return out


def tree_to_list(t):
    if t is None:
        return None
    return [t[0], t[1], t[2], t[3], t[4], tree_to_list(t[5]), tree_to_list(t[6])]


def _same_float(x, y):
    """Equal float32 bits, or both NaN.  NaN payloads differ between the
    reference's x86 build (default NaN 0xffc00000) and the GPU (0x7fffffff);
    Postgres never inspects them."""
    if math.isnan(x) or math.isnan(y):
        return math.isnan(x) and math.isnan(y)
    return struct.pack("<f", x) == struct.pack("<f", y)


def same_tree(a, b):
    """Bit-identical plan trees: ids, rows, costs, widths, shape."""
    if a is None or b is None:
        return a is None and b is None
    a = tree_to_list(a)
    b = tree_to_list(b)
    return (a[0] == b[0] and a[4] == b[4] and all(_same_float(a[i], b[i]) for i in (1, 2, 3))
            and same_tree(a[5], b[5]) and same_tree(a[6], b[6]))


@pytest.fixture(scope="session")
def golden_cases():
    return load_golden()
