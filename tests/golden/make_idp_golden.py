"""Golden fixtures of the IDP2 / UnionDP drivers, from the REFERENCE.

Each line of ``idp_cases.jsonl``: a seeded query, the IDP settings
(gpuqo_idp_n_iters, gpuqo_idp_type: 1 = IDP2, 2 = UNION), algorithm code 5
(GPUQO_CPU_DPSUB_BICC: MPDP sub-problems) and the plan the reference's
gpuqo_run returned (oracle/_ref/libgpuqo_ref.so, built from the reference's
sources by ``make -C oracle ref``).  The reference provides UnionDP only
below 64 relations (gpuqo_dpdp_union.cu instantiates it for Bitmapset32/64).

Usage: python tests/golden/make_idp_golden.py [--tags idp2_large --append]
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

IDP2, UNION = 1, 2


def cases():
    out = []
    for (q, k) in [(query.snowflake(30, 0), 10), (query.snowflake(40, 1), 15), (query.snowflake(60, 2), 25),
                   (query.snowflake(45, 3, rich=True), 12), (query.star(30, 4), 12), (query.chain(40, 5), 10),
                   (query.cycle(35, 6), 10), (query.random_graph(35, 7, extra_edge_p=0.05), 12),
                   (query.snowflake(80, 8), 12), (query.snowflake(150, 9), 15),
                   (query.random_graph(100, 10, extra_edge_p=0.01), 10)]:
        out.append(("idp2", q, k, IDP2))
    for (q, k) in [(query.snowflake(30, 11), 25), (query.snowflake(40, 12), 15), (query.snowflake(60, 13), 25),
                   (query.snowflake(50, 14, rich=True), 12), (query.star(30, 15), 12), (query.chain(40, 16), 10),
                   (query.cycle(35, 17), 10), (query.random_graph(40, 18, extra_edge_p=0.05), 12)]:
        out.append(("union", q, k, UNION))
    # the served workload's sizes (snowflakes of 30..1000 relations, k = 25):
    # the reference runs them on its dynamic bitsets
    for (q, k) in [(query.snowflake(300, 20), 25), (query.snowflake(1000, 21), 25)]:
        out.append(("idp2_large", q, k, IDP2))
    return out


def tree_json(t):
    if t is None:
        return None
    return [t[0], t[1], t[2], t[3], t[4], tree_json(t[5]), tree_json(t[6])]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tags", default="", help="comma-separated tags to generate (default: all)")
    ap.add_argument("--append", action="store_true", help="append to the fixture file instead of rewriting it")
    args = ap.parse_args()
    tags = set(t for t in args.tags.split(",") if t)
    if not harness.ref_available():
        sys.exit("oracle/_ref/libgpuqo_ref.so missing: run `make -C oracle ref` first")
    with open(os.path.join(HERE, "idp_cases.jsonl"), "a" if args.append else "w") as f:
        for tag, q, k, typ in cases():
            if tags and tag not in tags:
                continue
            t0 = time.time()
            tree, _ = harness.run_ref(q, 5, idp_n_iters=k, idp_type=typ)
            rec = {"tag": tag, "name": q.name, "algorithm": 5, "idp_n_iters": k, "idp_type": typ,
                   "query": q.to_dict(), "expected": tree_json(tree)}
            f.write(json.dumps(rec, separators=(",", ":")) + "\n")
            f.flush()
            print(f"{tag:6s} {q.name:22s} k={k:2d} {time.time() - t0:7.2f}s root_total={tree[3]!r}", flush=True)


if __name__ == "__main__":
    main()
