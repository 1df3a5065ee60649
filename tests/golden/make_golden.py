"""Generate the golden fixtures of the DP parity tests from the REFERENCE.

Each line of ``cases.jsonl`` holds one seeded synthetic query (the generators
of gpuqo_b200.query), the algorithm code, and the plan the reference's own
gpuqo_run returned for it -- oracle/_ref/libgpuqo_ref.so, the reference's
gpuqo module compiled from its sources by ``make -C oracle ref``.

Algorithm codes follow src/include/optimizer/gpuqo_common.h:13-29:
3 = GPUQO_CPU_DPSUB (plain DPsub), 5 = GPUQO_CPU_DPSUB_BICC (MPDP).

Usage (needs the reference library; run where the reference sources are):
    python tests/golden/make_golden.py            # small + full-size cases
    python tests/golden/make_golden.py --quick    # skip the minutes-long ones
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import harness  # noqa: E402
from gpuqo_b200 import query  # noqa: E402

DPSUB, BICC = 3, 5


def cases(quick):
    out = []
    # configuration 1: 12-relation star, plain DPsub
    for s in range(10):
        out.append(("star12", query.star(12, s), DPSUB))
    # configuration 2: 25-relation snowflake, MPDP
    for s in range(3):
        out.append(("snowflake25", query.snowflake(25, s), BICC))
    # configuration 3 at reduced sizes
    for s in range(3):
        out.append(("clique10", query.clique(10, s), DPSUB))
        out.append(("chain20", query.chain(20, s), DPSUB))
        out.append(("cycle20", query.cycle(20, s), DPSUB))
        out.append(("chain16_bicc", query.chain(16, s), BICC))
        out.append(("cycle16_bicc", query.cycle(16, s), BICC))
    out.append(("clique12", query.clique(12, 0), DPSUB))
    out.append(("clique12_bicc", query.clique(12, 0), BICC))
    # cost-model branches: statistics, unique indexes, multi-member classes
    for s in range(6):
        out.append(("random_rich", query.random_graph(8 + s, s, rich=True), DPSUB))
        out.append(("random_rich_bicc", query.random_graph(10 + s, s, extra_edge_p=0.25, rich=True), BICC))
        out.append(("equal_ties", query.random_graph(9, s, equal=True), DPSUB))
        out.append(("equal_ties_bicc", query.random_graph(11, s, equal=True), BICC))
        out.append(("multi_member", query.multi_member_classes(8 + s % 3, s), DPSUB))
        out.append(("multi_member_bicc", query.multi_member_classes(10 + s % 3, s), BICC))
    out.append(("star12_rich_bicc", query.star(12, 3, rich=True), BICC))
    out.append(("snowflake16_rich", query.snowflake(16, 4, rich=True), DPSUB))
    # edge sizes: a single relation and a single join
    out.append(("single", query.chain(1, 0), DPSUB))
    out.append(("pair", query.chain(2, 0), BICC))
    if not quick:
        # configuration 3 at full size (minutes of reference CPU time each)
        out.append(("clique14_bicc", query.clique(14, 0), BICC))
        out.append(("chain30", query.chain(30, 0), DPSUB))
        out.append(("cycle30", query.cycle(30, 0), DPSUB))
        out.append(("chain30_bicc", query.chain(30, 0), BICC))
        out.append(("cycle30_bicc", query.cycle(30, 0), BICC))
    return out


def tree_json(t):
    if t is None:
        return None
    return [t[0], t[1], t[2], t[3], t[4], tree_json(t[5]), tree_json(t[6])]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=os.path.join(HERE, "cases.jsonl"))
    args = ap.parse_args()
    if not harness.ref_available():
        sys.exit("oracle/_ref/libgpuqo_ref.so missing: run `make -C oracle ref` first")
    with open(args.out, "w") as f:
        for tag, q, alg in cases(args.quick):
            t0 = time.time()
            tree, _ = harness.run_ref(q, alg)
            rec = {"tag": tag, "name": q.name, "algorithm": alg,
                   "query": q.to_dict(), "expected": tree_json(tree)}
            f.write(json.dumps(rec, separators=(",", ":")) + "\n")
            f.flush()
            print(f"{tag:20s} {q.name:24s} alg={alg} {time.time() - t0:7.2f}s "
                  f"root_total={tree[3]!r}", flush=True)


if __name__ == "__main__":
    main()
