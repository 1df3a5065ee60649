import json
import os
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


def load_golden():
    from gpuqo_b200.query import Query
    out = []
    with open(GOLDEN) as f:
        for line in f:
            rec = json.loads(line)
            rec["query"] = Query.from_dict(rec["query"])
            out.append(rec)
    return out


def tree_to_list(t):
    if t is None:
        return None
    return [t[0], t[1], t[2], t[3], t[4], tree_to_list(t[5]), tree_to_list(t[6])]


def same_tree(a, b):
    """Bit-identical plan trees: ids, rows, costs, widths, shape."""
    return tree_to_list(a) == tree_to_list(b)


@pytest.fixture(scope="session")
def golden_cases():
    return load_golden()
