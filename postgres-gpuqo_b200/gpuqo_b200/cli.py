"""Plan seeded synthetic queries through the library from the command line.

    PYTHONPATH=postgres-gpuqo_b200 python -m gpuqo_b200.cli --shape snowflake --n 25 --repeat 2
    PYTHONPATH=postgres-gpuqo_b200 python -m gpuqo_b200.cli --shape star --n 12 --batch 4096

One line per call: wall time, device time, kernel launches and the counters of
the last call (gpuqo_b200_get_stats).  --batch K plans K queries of the shape
(seeds seed..seed+K-1) with one gpuqo_b200_run_batch call; --mix plans the
mixed workload of query.batch_mix (relation counts in [--nmin, --n]).
Also the fixed command used for profiler captures of single kernels.
"""
import argparse
import ctypes as C
import time

from . import capi, lib, query

ALGS = {"mpdp": (capi.GPUQO_DPSUB, True), "dpsub": (capi.GPUQO_DPSUB, False)}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m gpuqo_b200.cli")
    ap.add_argument("--shape", default="snowflake", choices=sorted(query.SHAPES),
                    help="query graph; key_chain, key_cycle, lollipop and ring_path reach 63 relations "
                         "(the sparse exact DP beyond 31)")
    ap.add_argument("--n", type=int, default=25)
    ap.add_argument("--nmin", type=int, default=8)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--alg", default="mpdp", choices=sorted(ALGS))
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--batch", type=int, default=0, help="queries per gpuqo_b200_run_batch call (0: gpuqo_run)")
    ap.add_argument("--mix", action="store_true", help="batch of the mixed workload instead of one shape")
    ap.add_argument("--idp", type=int, default=0, help="gpuqo_idp_n_iters (IDP2 when > 1)")
    ap.add_argument("--persistent", type=int, default=1, help="gpuqo_b200_persistent")
    ap.add_argument("--autotune", action="store_true", help="run gpuqo_b200_autotune first")
    ap.add_argument("--tuning", default=None, metavar="NARROW,WIDE,HANDOFF",
                    help="install these crossovers instead (gpuqo_b200_set_tuning): connected sets per level up to "
                         "which the 2-blocks tree kernel runs, above which the 4-blocks one runs, and the batch "
                         "hand-off in connected sets")
    a = ap.parse_args(argv)

    L = lib.load()
    alg, bicc = ALGS[a.alg]
    capi.set_bool(L, "gpuqo_dpsub_bicc_enable", bicc)
    capi.set_int(L, "gpuqo_idp_n_iters", a.idp)
    capi.set_int(L, "gpuqo_idp_type", capi.GPUQO_IDP2)
    capi.set_int(L, "gpuqo_b200_persistent", a.persistent)
    if a.autotune:
        print("tuning:", lib.autotune(), flush=True)
    if a.tuning:
        lib.set_tuning(*[float(x) for x in a.tuning.split(",")])
        print("tuning:", lib.get_tuning(), flush=True)
    if a.batch:
        qs = (query.batch_mix(a.batch, seed=a.seed, nmin=a.nmin, nmax=a.n) if a.mix else
              [query.make(a.shape, a.n, a.seed + i) for i in range(a.batch)])
    else:
        qs = [query.make(a.shape, a.n, a.seed)]
    builders = [capi.PlannerInfoBuilder(q) for q in qs]
    arr = (C.POINTER(capi.GpuqoPlannerInfoC) * len(qs))(*[b.pointer() for b in builders])
    out = (C.POINTER(capi.QueryTreeC) * len(qs))()
    for r in range(a.repeat):
        t = time.perf_counter()
        if a.batch:
            rc = L.gpuqo_b200_run_batch(alg, arr, len(qs), out)
        else:
            out[0] = L.gpuqo_run(alg, builders[0].pointer())
            rc = 0 if out[0] else L.gpuqo_b200_last_error()
        dt = time.perf_counter() - t
        st = lib.get_stats()
        for i in range(len(qs)):
            if out[i]:
                L.gpuqo_b200_free_query_tree(C.cast(out[i], C.c_void_p))
                out[i] = None
        print(f"call {r}: rc={rc} wall {dt * 1e3:.3f} ms device {st['device_ms']:.3f} ms "
              f"launches {st['kernel_launches']} sets {st['connected_sets']} pairs {st['evaluated_pairs']}",
              flush=True)
        if rc:
            raise SystemExit(rc)


if __name__ == "__main__":
    main()
