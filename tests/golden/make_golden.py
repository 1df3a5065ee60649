"""Generate the golden fixtures of the DP parity tests from the REFERENCE.

Each line of ``cases.jsonl`` holds one seeded synthetic query (the generators
of gpuqo_b200.query), the algorithm code, and the plan the reference's own
gpuqo_run returned for it -- oracle/_ref/libgpuqo_ref.so, the reference's
gpuqo module compiled from its sources by ``make -C oracle ref``.

Algorithm codes follow src/include/optimizer/gpuqo_common.h:13-29:
3 = GPUQO_CPU_DPSUB (plain DPsub), 5 = GPUQO_CPU_DPSUB_BICC (MPDP).

``spanning_cases.jsonl`` (``--spanning``) holds queries planned with
gpuqo_spanning_tree_enable set: the reference replaces the join graph by its
minimum spanning tree before any algorithm runs (exact DP or IDP).
``dpsize_cases.jsonl`` (``--dpsize``) holds the plans of the reference's
cpu_dpsize (algorithm code 2), the tie order the library's DPsize follows.
``wide_cases.jsonl`` (``--wide``) holds cpu_dpccp (code 7) plans of 32 to 63
relations, the optimum the sparse exact DP must reach.

Usage (needs the reference library; run where the reference sources are):
    python tests/golden/make_golden.py            # small + full-size cases
    python tests/golden/make_golden.py --quick    # skip the minutes-long ones
    python tests/golden/make_golden.py --spanning # the spanning-tree fixtures
    python tests/golden/make_golden.py --dpsize   # the DPsize fixtures
    python tests/golden/make_golden.py --wide     # the 32-63 relation fixtures
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
    for s in range(4):
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
        out.append(("clique18", query.clique(18, 0), DPSUB))
        out.append(("chain30", query.chain(30, 0), DPSUB))
        out.append(("cycle30", query.cycle(30, 0), DPSUB))
        out.append(("chain30_bicc", query.chain(30, 0), BICC))
        out.append(("cycle30_bicc", query.cycle(30, 0), BICC))
    return out


def spanning_cases():
    """(tag, query, algorithm, idp_n_iters, idp_type) with the spanning tree on."""
    out = []
    for s in range(4):
        out.append(("sp_random", query.random_graph(9 + s, 9100 + s, extra_edge_p=0.35, rich=True), DPSUB, 0, 1))
        out.append(("sp_random_bicc", query.random_graph(11 + s, 9200 + s, extra_edge_p=0.35, rich=True), BICC, 0, 1))
        out.append(("sp_multi", query.multi_member_classes(9 + s, 9300 + s), BICC, 0, 1))
    out.append(("sp_cycle", query.cycle(14, 9400), BICC, 0, 1))
    out.append(("sp_clique", query.clique(9, 9401), DPSUB, 0, 1))
    out.append(("sp_clique_bicc", query.clique(10, 9402, rich=True), BICC, 0, 1))
    out.append(("sp_equal", query.random_graph(10, 9403, extra_edge_p=0.4, equal=True), BICC, 0, 1))
    # IDP2 over the spanning tree, 64-bit and dynamic relation sets
    out.append(("sp_idp2", query.random_graph(40, 9500, extra_edge_p=0.06), BICC, 12, 1))
    out.append(("sp_idp2_dyn", query.random_graph(80, 9501, extra_edge_p=0.03), BICC, 12, 1))
    out.append(("sp_union", query.random_graph(36, 9502, extra_edge_p=0.06), BICC, 10, 2))
    return out


def dpsize_cases():
    """(tag, query, algorithm, idp_n_iters, idp_type) for cpu_dpsize (code 2)."""
    DPSIZE = 2
    out = []
    for s in range(3):
        out.append(("dz_star12", query.star(12, s), DPSIZE, 0, 1))
        out.append(("dz_snowflake16", query.snowflake(16, 9600 + s), DPSIZE, 0, 1))
        out.append(("dz_random", query.random_graph(11 + s, 9610 + s, extra_edge_p=0.3, rich=True), DPSIZE, 0, 1))
        out.append(("dz_equal", query.random_graph(10 + s, 9620 + s, extra_edge_p=0.3, equal=True), DPSIZE, 0, 1))
        out.append(("dz_multi", query.multi_member_classes(9 + s, 9630 + s), DPSIZE, 0, 1))
    out.append(("dz_chain18", query.chain(18, 9640), DPSIZE, 0, 1))
    out.append(("dz_cycle14", query.cycle(14, 9641), DPSIZE, 0, 1))
    out.append(("dz_clique9", query.clique(9, 9642), DPSIZE, 0, 1))
    out.append(("dz_single", query.chain(1, 0), DPSIZE, 0, 1))
    out.append(("dz_pair", query.chain(2, 1), DPSIZE, 0, 1))
    out.append(("dz_idp2", query.snowflake(40, 9650), DPSIZE, 10, 1))
    return out


def wide_cases():
    """(tag, query, algorithm, idp_n_iters, idp_type) of 32 to 63 relations,
    planned by the reference's cpu_dpccp (code 7): the reference's only exact
    DP that finishes at these sizes (its DPsub and MPDP visit all 2^n subsets
    of the relations).  The fixtures pin the optimum (root rows and total
    cost) of the sparse exact DP, whose tie order is DPsub's or MPDP's."""
    DPCCP = 7
    return [("wide_key_chain32", query.key_chain(32, 11), DPCCP, 0, 1),
            ("wide_key_chain40", query.key_chain(40, 1), DPCCP, 0, 1),
            ("wide_key_chain63", query.key_chain(63, 4), DPCCP, 0, 1),
            ("wide_key_cycle40", query.key_cycle(40, 2), DPCCP, 0, 1),
            ("wide_key_cycle48_rich", query.key_cycle(48, 8, rich=True), DPCCP, 0, 1),
            ("wide_key_cycle63", query.key_cycle(63, 5), DPCCP, 0, 1),
            ("wide_lollipop40", query.lollipop(40, 4), DPCCP, 0, 1),
            ("wide_lollipop63_rich", query.lollipop(63, 7, rich=True), DPCCP, 0, 1),
            ("wide_ring_path40", query.ring_path(40, 3), DPCCP, 0, 1),
            ("wide_ring_path36_rich", query.ring_path(36, 10, rich=True), DPCCP, 0, 1),
            # the snowflake workload beyond the dense memo: 1.2 M and 2.4 M connected sets
            ("wide_snowflake32", query.snowflake(32, 1), DPCCP, 0, 1),
            ("wide_snowflake34", query.snowflake(34, 5), DPCCP, 0, 1)]


def tree_json(t):
    if t is None:
        return None
    return [t[0], t[1], t[2], t[3], t[4], tree_json(t[5]), tree_json(t[6])]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=os.path.join(HERE, "cases.jsonl"))
    ap.add_argument("--spanning", action="store_true", help="write spanning_cases.jsonl instead")
    ap.add_argument("--dpsize", action="store_true", help="write dpsize_cases.jsonl (cpu_dpsize) instead")
    ap.add_argument("--wide", action="store_true", help="write wide_cases.jsonl (cpu_dpccp, 32-63 relations)")
    args = ap.parse_args()
    if not harness.ref_available():
        sys.exit("oracle/_ref/libgpuqo_ref.so missing: run `make -C oracle ref` first")
    if args.spanning or args.dpsize or args.wide:
        fname, gen = (("spanning_cases.jsonl", spanning_cases) if args.spanning else
                      ("wide_cases.jsonl", wide_cases) if args.wide else ("dpsize_cases.jsonl", dpsize_cases))
        with open(os.path.join(HERE, fname), "w") as f:
            for tag, q, alg, k, typ in gen():
                t0 = time.time()
                tree, _ = harness.run_ref(q, alg, idp_n_iters=k, idp_type=typ, spanning=args.spanning)
                rec = {"tag": tag, "name": q.name, "algorithm": alg, "idp_n_iters": k, "idp_type": typ,
                       "query": q.to_dict(), "expected": tree_json(tree)}
                f.write(json.dumps(rec, separators=(",", ":")) + "\n")
                f.flush()
                print(f"{tag:16s} {q.name:24s} alg={alg} k={k} {time.time() - t0:7.2f}s root_total={tree[3]!r}",
                      flush=True)
        return
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
