"""Benchmark of the B200 join-order DP (MPDP on the 25-relation snowflake).

One step = one MPDP optimisation (gpuqo_algorithm=dpsub, gpuqo_dpsub_bicc=on)
of one seeded synthetic 25-relation snowflake query per rank.  Multi-GPU runs
are weak-scaled query sharding: every rank optimises its own queries, no
collective on the data path; the barrier and the max-over-ranks timing are
the only collectives.

Printed (rank 0, one JSON line):
  value  - ms per query of the device-resident DP: the planner info is on the
           device, the DP runs as one persistent cooperative launch
           (k_dp_tree: every level's enumeration and evaluation, grid
           barrier between levels), CUDA events on the library's stream, L2
           flushed (256 MB write) before every step;
  e2e    - ms per query through the C ABI gpuqo_run with host structures
           (conversion, H2D of the planner info, the DP, D2H of the plan);
  roofline - k_dp_tree: algorithmic memo bytes per launch (32 B per
           evaluated csg-cmp pair: two 16 B memo reads; 20 B per connected set
           written) over its event-timed launch duration, against the
           measured HBM copy bandwidth;
  cpu_baseline - the reference's parallel_cpu_dpsub_bicc (its own code,
           compiled from its sources into oracle/_ref) on the host cores,
           median of at least 5 runs after a warm-up, with the CPU model;
  configs  - configurations 1 and 3: plain DPsub (gpuqo_dpsub_bicc off) on
           the 12-relation stars, the 18-relation clique and the 30-relation
           chain and cycle, device-resident ms/query and evaluated pairs/s,
           each plan compared bit for bit with the reference's golden plan
           (tests/golden/cases.jsonl); beside them the reference's dpe_dpsub
           and cpu_dpsub on the stars (host cores), and the -march=native
           build of the reference where this CPU can run it;
  batched - 4096 queries of the mixed workload (40% star, 40% snowflake, 10%
           chain, 10% cycle; relation counts uniform in [8,28], and [8,16])
           through gpuqo_b200_run_batch against gpuqo_run one query per call,
           queries per second and a bit-for-bit plan comparison;
  served - IDP2 and UnionDP (k=25) snowflake queries of 30..1000 relations
           arriving as a Poisson stream at 1x and 4x the plain capacity
           (UnionDP also 8x and 16x) into
           the continuous-batching service: queries/s, p50/p99 latency,
           against one-at-a-time gpuqo_run served first-in first-out under
           the same arrivals (a worker thread, measured).

--impl reference times that reference CPU engine alone (rank 0 only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "postgres-gpuqo_b200"))

METRIC = "MPDP ms/query @25-rel snowflake; batched queries/s vs plain GPU; p50/p99"
WORKLOAD = ("MPDP (gpuqo_algorithm=dpsub, gpuqo_dpsub_bicc=on) of one 25-relation snowflake "
            "query per step: root with 4-6 children, 0-3 children per node, depth <= 4, rows "
            "log-uniform [1e2,1e8], FK-PK selectivity 1/rows(PK side), dense memo 2^25")
N_RELS = 25
SEEDS = [0, 1, 2, 3]


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seeds(rank):
    """This rank's query seeds: every rank optimises its own queries (weak
    scaling, no data-path collective)."""
    return [s + 1000 * rank for s in SEEDS]


def max_over_ranks(x, dist, device):
    """The largest of every rank's x (device time of the timed region)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_ms_per_query(max_ms, steps, world):
    """All ranks optimised steps queries each within max_ms."""
    return max_ms / (steps * world)


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_figure(key):
    """A figure of profiles/k_dp_tree_snowflake25_traffic.txt (the ncu
    captures of this benchmark's own workload): dram_bytes_per_launch (DRAM
    read + write per timed k_dp_tree launch, the four snowflake-25 seeds),
    l2_throughput_pct_of_peak or issue_active_pct; None when absent."""
    p = os.path.join(REPO, "profiles", "k_dp_tree_snowflake25_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock and clock-event reasons sampled DURING the timed region: an
    NVML poller thread reads them every 2 ms (the timed regions are only a
    few milliseconds long); where NVML is not available, nvidia-smi every
    100 ms.  Reading clocks changes no GPU setting."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []          # (sm_mhz, max_mhz, reasons bitmask)
        self.stop = threading.Event()
        self.t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            hnd = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(hnd, pynvml.NVML_CLOCK_SM)

            def poll():
                while not self.stop.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(hnd, pynvml.NVML_CLOCK_SM)
                        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(hnd)
                        self.samples.append((float(sm), float(mx), int(rs)))
                    except Exception:
                        pass
                    self.stop.wait(0.002)
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.samples = []
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        elif self.t is not None:
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        for s_mhz, m_mhz, bits in self.samples:
            sm.append(s_mhz)
            mx.append(m_mhz)
            for nm, bit in self.REASONS:
                if bits & bit:
                    reasons.add(nm)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference_sample(queries, algorithm, steps=None, budget_s=20.0, min_runs=5, max_runs=40, native=False,
                         threads=None):
    """The reference's own CPU engine (oracle/_ref, or its -march=native
    build) on the host cores: one warm-up, then at least min_runs timed calls
    (steady clock around gpuqo_run) within about budget_s; returns the median
    and mean ms per query, the threads used and the number of runs."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import harness
    cores = threads or os.cpu_count() or 1
    harness.run_ref(queries[0], algorithm, threads=cores, native=native)   # warm-up
    times = []
    t_start = time.perf_counter()
    i = 0
    while True:
        q = queries[i % len(queries)]
        _, dt = harness.run_ref(q, algorithm, threads=cores, native=native)
        times.append(dt * 1000.0)
        i += 1
        if steps is not None:
            if i >= steps:
                break
        elif i >= max_runs or (i >= min_runs and time.perf_counter() - t_start > budget_s):
            break
    return statistics.median(times), statistics.mean(times), cores, len(times)


GOLDEN = os.path.join(REPO, "tests", "golden", "cases.jsonl")


def golden_cases(tag, algorithm, path=GOLDEN):
    """The committed golden queries of one tag with the reference's plans."""
    from gpuqo_b200.query import Query
    out = []
    with open(path) as f:
        for line in f:
            rec = json.loads(line)
            if rec["tag"] == tag and rec["algorithm"] == algorithm:
                rec["query"] = Query.from_dict(rec["query"])
                out.append(rec)
    return out


def configs_section(cpu=True):
    """Configurations 1 and 3 (plain DPsub): device-resident time of each
    golden query (L2 flushed before every replay), evaluated pairs/s, and a
    bit-for-bit comparison with the reference's golden plan; the reference's
    CPU engines on the configuration-1 stars beside them."""
    from gpuqo_b200 import capi, lib
    res = {}
    for tag, what in (("star12", "12-relation stars (configuration 1), seeds 0-9"),
                      ("clique18", "18-relation clique (configuration 3)"),
                      ("chain30", "30-relation chain (configuration 3)"),
                      ("cycle30", "30-relation cycle (configuration 3)")):
        cases = golden_cases(tag, capi.GPUQO_CPU_DPSUB)
        if not cases:
            continue
        ms_all, pairs, csgs, same, launches = [], 0, 0, True, 0
        for c in cases:
            rc, ms, tree, st = lib.time_resident(c["query"], capi.GPUQO_DPSUB, bicc=False, warmup=2, iters=5,
                                                 flush_l2=True)
            if rc or tree is None:
                raise RuntimeError(f"gpuqo_b200_time_resident failed on {c['name']}: {rc}")
            ms_all.append(ms)
            pairs += st["evaluated_pairs"]
            csgs += st["connected_sets"]
            launches = max(launches, st["kernel_launches"])
            same = same and capi.same_plan(tree, c["expected"])
        tot = sum(ms_all)
        res[tag] = {"workload": what, "queries": len(cases), "ms_per_query": tot / len(cases),
                    "evaluated_pairs_per_query": pairs / len(cases), "connected_sets_per_query": csgs / len(cases),
                    "pairs_per_s": pairs / (tot / 1000.0) if tot > 0 else None,
                    "kernel_launches_per_query": launches, "identical_plans_vs_reference": same}
    if cpu and "star12" in res:
        qs = [c["query"] for c in golden_cases("star12", capi.GPUQO_CPU_DPSUB)]
        cores = os.cpu_count() or 1
        base = {}
        for name, alg, thr in (("dpe_dpsub", capi.GPUQO_DPE_DPSUB, cores),
                               ("cpu_dpsub", capi.GPUQO_CPU_DPSUB, 1)):
            med, mean, used, nr = cpu_reference_sample(qs, alg, budget_s=5.0, threads=thr)
            base[name] = {"median_ms_per_query": med, "mean_ms_per_query": mean, "threads": used, "runs": nr}
        ok, why = native_reference_usable()
        if ok:
            med, mean, used, nr = cpu_reference_sample(qs, capi.GPUQO_DPE_DPSUB, budget_s=5.0, native=True)
            base["dpe_dpsub_march_native"] = {"median_ms_per_query": med, "mean_ms_per_query": mean,
                                              "threads": used, "runs": nr}
        else:
            base["dpe_dpsub_march_native"] = {"skipped": why}
        res["star12"]["reference_cpu"] = base
        res["star12"]["reference_cpu_note"] = ("the reference's own engines (oracle/_ref) on the same stars: "
                                               "dpe_dpsub with gpuqo_dpe_n_threads = all host threads and "
                                               "gpuqo_dpe_pairs_per_depbuf 65536, cpu_dpsub on one thread")
    res.update(wide_section(cpu))
    return res


WIDE_GOLDEN = os.path.join(REPO, "tests", "golden", "wide_cases.jsonl")


def wide_section(cpu=True):
    """Exact MPDP of 40 to 63 relations on the sparse memo, through gpuqo_run
    from host structures (wall time and device time), with the root's rows
    and total cost against the optimum of the reference's cpu_dpccp (the
    committed fixtures), and that engine's own time on the same query."""
    from gpuqo_b200 import capi, lib
    res = {}
    for tag in ("wide_key_chain63", "wide_key_cycle63", "wide_lollipop63_rich", "wide_ring_path40",
                "wide_snowflake32", "wide_snowflake34"):
        cases = golden_cases(tag, capi.GPUQO_CPU_DPCCP, WIDE_GOLDEN)
        if not cases:
            continue
        c = cases[0]
        q = c["query"]
        lib.run(q, capi.GPUQO_DPSUB, bicc=True)                          # warm-up
        wall, dev = [], []
        for _ in range(5):
            r = lib.run(q, capi.GPUQO_DPSUB, bicc=True)
            if r.error or r.tree is None:
                raise RuntimeError(f"sparse exact DP failed on {q.name}: {r.error}")
            wall.append(r.seconds * 1000.0)
            dev.append(r.stats["device_ms"])
        entry = {"workload": f"{q.n}-relation {q.name.rsplit('_s', 1)[0].rstrip('0123456789')} (MPDP, sparse memo)",
                 "ms_per_query_wall": statistics.median(wall), "device_ms": statistics.median(dev),
                 "connected_sets": r.stats["connected_sets"], "evaluated_pairs": r.stats["evaluated_pairs"],
                 "kernel_launches": r.stats["kernel_launches"],
                 "reference_optimum_reached": r.tree[3] == c["expected"][3]}
        if cpu and not tag.startswith("wide_snowflake"):   # cpu_dpccp takes 40-90 s on those
            med, mean, used, nr = cpu_reference_sample([q], capi.GPUQO_CPU_DPCCP, budget_s=3.0, threads=1)
            entry["reference_cpu_dpccp"] = {"median_ms_per_query": med, "threads": used, "runs": nr,
                                            "note": "the reference's exact DP that runs at this size; its DPsub "
                                                    "and MPDP visit all 2^n subsets"}
        res[tag.replace("wide_", "wide:")] = entry
    return res


def native_reference_usable():
    """The -march=native build of the reference runs only on a CPU with every
    ISA extension of the machine that built it."""
    lib = os.path.join(REPO, "oracle", "_ref", "libgpuqo_ref_native.so")
    isa = os.path.join(REPO, "oracle", "_ref", "libgpuqo_ref_native.isa")
    if not (os.path.exists(lib) and os.path.exists(isa)):
        return False, "not built"
    need = set(open(isa).read().split())
    have = set()
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                have = set(line.split(":", 1)[1].split())
                break
    except OSError:
        return False, "no /proc/cpuinfo"
    missing = sorted(need - have)
    if missing:
        return False, "this CPU lacks " + " ".join(missing[:6])
    return True, ""


def _prebuilt(qs):
    import ctypes as C
    from gpuqo_b200 import capi
    bs = [capi.PlannerInfoBuilder(q) for q in qs]
    arr = (C.POINTER(capi.GpuqoPlannerInfoC) * len(qs))(*[b.pointer() for b in bs])
    return bs, arr


def batched_section(seed=7):
    """Batched MPDP (gpuqo_b200_run_batch) against the plain one-query-per-call
    gpuqo_run on the same prebuilt planner infos; wall clock around the C
    calls (host conversion, H2D, DP, D2H, plan output all included), plans
    compared bit for bit."""
    import ctypes as C
    from gpuqo_b200 import capi, lib, query
    L = lib.load()
    capi.set_bool(L, "gpuqo_dpsub_bicc_enable", True)
    capi.set_int(L, "gpuqo_idp_n_iters", 0)

    def run_batch(arr, m):
        out = (C.POINTER(capi.QueryTreeC) * m)()
        t = time.perf_counter()
        rc = L.gpuqo_b200_run_batch(capi.GPUQO_DPSUB, arr, m, out)
        dt = time.perf_counter() - t
        st = lib.get_stats()
        trees = [capi.tree_to_py(out[i]) for i in range(m)]
        for i in range(m):
            L.gpuqo_b200_free_query_tree(C.cast(out[i], C.c_void_p))
        if rc:
            raise RuntimeError(f"gpuqo_b200_run_batch failed: {rc}")
        return dt, st, trees

    res = {}
    for tag, nmin, nmax in (("n8_28", 8, 28), ("n8_16", 8, 16)):
        qs = query.batch_mix(4096, seed=seed, nmin=nmin, nmax=nmax)
        bs, arr = _prebuilt(qs)
        _, warr = _prebuilt(query.batch_mix(64, seed=seed + 1, nmin=nmin, nmax=min(nmax, 20)))
        run_batch(warr, 64)                                  # warm-up (engines, arenas)
        if nmax > 20:
            # the full mix once more untimed: its largest queries and waves
            # size the device memos and arenas, which the plain arm after it
            # then finds allocated too
            run_batch(arr, len(qs))
        # the short batches (host-heavy: tens of ms) take the median of three
        # runs; the long one runs once
        runs = [run_batch(arr, len(qs)) for _ in range(3 if nmax <= 20 else 1)]
        runs.sort(key=lambda x: x[0])
        dtb, st, trees = runs[len(runs) // 2]
        t = time.perf_counter()
        same = True
        for b, tb in zip(bs, trees):
            r = L.gpuqo_run(capi.GPUQO_DPSUB, b.pointer())
            same = same and capi.same_plan(capi.tree_to_py(r), tb)
            L.gpuqo_b200_free_query_tree(C.cast(r, C.c_void_p))
        dtp = time.perf_counter() - t
        hand = st.get("handoff_device_ms", 0.0)
        res[tag] = {"queries": len(qs), "batched_runs": len(runs), "batched_qps": len(qs) / dtb,
                    "plain_qps": len(qs) / dtp,
                    "speedup": dtp / dtb, "batched_device_ms": st["device_ms"],
                    "batched_launches": st["kernel_launches"], "identical_plans": same,
                    # the queries that fill the GPU alone run in the same
                    # single-query kernel in both arms: no batching can make the
                    # batch faster than their device time, so plain time over
                    # it bounds the speedup
                    "handoff_device_ms": hand,
                    "speedup_bound": (dtp * 1000.0 / hand) if hand > 0 else None}
    return {"workload": "4096 MPDP queries, shapes 40% star / 40% snowflake / 10% chain / 10% cycle, "
                        "relation counts uniform in the range (n8_28: the full [8,28] mix; n8_16: small queries)",
            "arms": "batched = gpuqo_b200_run_batch of all queries (waves of one cooperative launch each); "
                    "plain = gpuqo_run per query; both from host planner infos to palloc'd plans",
            "by_range": res}


def served_section(n_req=192, seed=5):
    """Served IDP2 and UnionDP (k=25) over MPDP: Poisson arrivals of snowflake
    queries with relation counts log-uniform in [30,1000] into the
    continuous-batching service, against one-at-a-time plain gpuqo_run run
    by a first-in first-out worker thread under the same arrivals (both arms
    measured with the wall clock from each request's arrival).  The stream is
    long enough (192 requests) that the throughput is the steady state's, not
    the latency of the last large request after the arrivals end."""
    import ctypes as C
    import math
    import threading
    import numpy as np
    from gpuqo_b200 import capi, lib, query
    rng = np.random.default_rng(seed)
    ns = [int(round(math.exp(rng.uniform(math.log(30), math.log(1000))))) for _ in range(n_req)]
    qs = [query.snowflake(n, 9000 + i) for i, n in enumerate(ns)]
    L = lib.load()
    capi.set_bool(L, "gpuqo_dpsub_bicc_enable", True)
    capi.set_int(L, "gpuqo_idp_n_iters", 25)
    builders = [capi.PlannerInfoBuilder(q) for q in qs]
    out = {"workload": f"{n_req} snowflake queries, relation counts log-uniform in [30,1000], gpuqo_idp_n_iters=25 "
                       f"over MPDP, Poisson arrivals at 1x and 4x the plain capacity (UnionDP, which keeps "
                       f"up with 4x, also at 8x and 16x)", "by_idp_type": {}}
    for idp_type, tag in ((capi.GPUQO_IDP2, "idp2"), (capi.GPUQO_UNION, "union")):
        capi.set_int(L, "gpuqo_idp_type", idp_type)
        r = L.gpuqo_run(capi.GPUQO_DPSUB, builders[0].pointer())   # warm-up
        L.gpuqo_b200_free_query_tree(C.cast(r, C.c_void_p))
        svc, plain = [], []
        for b in builders:
            t = time.perf_counter()
            r = L.gpuqo_run(capi.GPUQO_DPSUB, b.pointer())
            svc.append(time.perf_counter() - t)
            plain.append(capi.tree_to_py(r))
            L.gpuqo_b200_free_query_tree(C.cast(r, C.c_void_p))
        plain_qps = n_req / sum(svc)
        res_t = {"plain_qps": plain_qps, "plain_mean_service_ms": 1e3 * sum(svc) / n_req, "rates": []}
        for mult in ((1.0, 4.0) if tag == "idp2" else (1.0, 4.0, 8.0, 16.0)):
            rate = plain_qps * mult
            arr = np.cumsum(rng.exponential(1.0 / rate, n_req))
            # plain arm, measured: one worker thread takes the requests in
            # arrival order and runs gpuqo_run on each (one query per call);
            # the plans are kept as returned and compared after the stream, so
            # the arm pays no Python conversion between two calls
            lats, trees = [0.0] * n_req, [None] * n_req
            t0 = time.perf_counter()

            def fifo_worker():
                for j in range(n_req):
                    now = time.perf_counter() - t0
                    if arr[j] > now:
                        time.sleep(arr[j] - now)
                    trees[j] = L.gpuqo_run(capi.GPUQO_DPSUB, builders[j].pointer())
                    lats[j] = time.perf_counter() - t0 - arr[j]
            w = threading.Thread(target=fifo_worker)
            w.start()
            w.join()
            fifo_makespan = time.perf_counter() - t0
            plain_same = [all(capi.same_plan(capi.tree_to_py(r), p) for r, p in zip(trees, plain))]
            for r in trees:
                L.gpuqo_b200_free_query_tree(C.cast(r, C.c_void_p))
            srv = lib.Server(max_inflight=32, wave_memory_mb=32768)
            res = [None] * n_req

            # the waiters keep the plans as returned; they are converted and
            # compared after the stream, as in the plain arm
            def waiter(j, tk):
                res[j] = srv.wait_raw(tk)
            ths = []
            t0 = time.perf_counter()
            for j in range(n_req):
                now = time.perf_counter() - t0
                if arr[j] > now:
                    time.sleep(arr[j] - now)
                tk = srv.submit_built(builders[j], capi.GPUQO_DPSUB)
                th = threading.Thread(target=waiter, args=(j, tk))
                th.start()
                ths.append(th)
            for th in ths:
                th.join()
            makespan = time.perf_counter() - t0
            st = srv.stats()
            srv.stop()
            served_same = all(rc == 0 and bool(r) and capi.same_plan(capi.tree_to_py(r), p)
                              for (rc, r, _), p in zip(res, plain))
            for _, r, _ in res:
                if r:
                    L.gpuqo_b200_free_query_tree(C.cast(r, C.c_void_p))
            lat = [x[2] for x in res]
            res_t["rates"].append({
                "arrival_qps": rate, "served_qps": n_req / makespan,
                "served_p50_ms": float(np.percentile(lat, 50)), "served_p99_ms": float(np.percentile(lat, 99)),
                "plain_fifo_p50_ms": 1e3 * float(np.percentile(lats, 50)),
                "plain_fifo_p99_ms": 1e3 * float(np.percentile(lats, 99)),
                "plain_fifo_qps": n_req / fifo_makespan,
                "plain_fifo_same_plans": plain_same[0],
                "identical_plans": served_same,
                "waves": st["waves"], "batched_subproblems": st["batched_subproblems"],
                "device_ms": st["device_ms"], "busy_ms": st["busy_ms"], "starved_ms": st["starved_ms"],
                # the service runs the same exact DPs on the device; at best it
                # hides all host work behind them, so the plain service time over
                # the device time per request bounds its gain
                "speedup_bound": (res_t["plain_mean_service_ms"] * n_req / st["device_ms"])
                                 if st["device_ms"] > 0 else None})
        out["by_idp_type"][tag] = res_t
    capi.set_int(L, "gpuqo_idp_n_iters", 0)
    capi.set_int(L, "gpuqo_idp_type", capi.GPUQO_IDP2)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (4096-query) section")
    ap.add_argument("--no-served", action="store_true", help="skip the served IDP2 section")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the configuration 1 and 3 section (plain DPsub on star-12, clique-18, chain-30, cycle-30)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in kernel-variant crossovers (for runs under a profiler, which distorts "
                         "the tuner's timings)")
    args = ap.parse_args()
    rank, world, local_rank = dist_env()

    from gpuqo_b200 import capi, query

    if args.impl == "reference":
        if rank != 0:
            return
        qs = [query.snowflake(N_RELS, s) for s in SEEDS]
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import harness
        cores = os.cpu_count() or 1
        for i in range(args.warmup):
            harness.run_ref(qs[i % len(qs)], capi.GPUQO_CPU_DPSUB_BICC_PARALLEL, threads=cores)
        times = []
        for i in range(args.steps):
            _, dt = harness.run_ref(qs[i % len(qs)], capi.GPUQO_CPU_DPSUB_BICC_PARALLEL, threads=cores)
            times.append(dt * 1000.0)
        v = statistics.mean(times)
        med = statistics.median(times)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ms/query", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "seeds": SEEDS, "engine": "parallel_cpu_dpsub_bicc",
                           "chunk": 256},
                "cpu_baseline": {"value": v, "unit": "ms/query", "cores": cores, "kind": "reference",
                                 "median": med, "cpu_model": cpu_model(),
                                 "sample": f"{args.steps} snowflake-25 queries, gpuqo_dpe_n_threads={cores}"},
                "e2e": {"value": v, "unit": "ms/query", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    from gpuqo_b200 import lib
    lib.load()
    # kernel-variant and batch hand-off crossovers of this device (about a second)
    tuning = lib.get_tuning() if args.no_autotune else lib.autotune()
    qs = [query.snowflake(N_RELS, s) for s in rank_seeds(rank)]

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (also captures the DP graph)
    for i in range(args.warmup):
        rc, _, _, _ = lib.time_resident(qs[i % len(qs)], capi.GPUQO_DPSUB, bicc=True, warmup=0, iters=1)
        if rc:
            raise RuntimeError(f"gpuqo_b200_time_resident failed: {rc}")

    # ---- timed region: device-resident DP ----
    tot_ms = 0.0
    eval_ms = 0.0
    eval_launches = 0
    kernels = 0
    pairs = 0
    csgs = 0
    barrier()
    with ClockSampler(local_rank) as clk:
        for i in range(args.steps):
            rc, ms, tree, st = lib.time_resident(qs[i % len(qs)], capi.GPUQO_DPSUB, bicc=True,
                                                 warmup=0, iters=1, flush_l2=True)
            if rc or tree is None:
                raise RuntimeError(f"gpuqo_b200_time_resident failed: {rc}")
            tot_ms += ms
            eval_ms += st["eval_kernel_ms"]
            eval_launches += st["eval_kernel_launches"]
            kernels += st["kernel_launches"]
            pairs += st["evaluated_pairs"]
            csgs += st["connected_sets"]
    barrier()
    max_ms = max_over_ranks(tot_ms, dist, "cuda")
    value = whole_job_ms_per_query(max_ms, args.steps, world)

    # ---- e2e: the C ABI with host structures ----
    for i in range(args.warmup):
        lib.run(qs[i % len(qs)], capi.GPUQO_DPSUB, bicc=True)
    barrier()
    e2e_ms = 0.0
    for i in range(args.steps):
        r = lib.run(qs[i % len(qs)], capi.GPUQO_DPSUB, bicc=True)
        if r.error or r.tree is None:
            raise RuntimeError(f"gpuqo_run failed: {r.error}")
        e2e_ms += r.seconds * 1000.0
    barrier()
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")
    e2e_value = whole_job_ms_per_query(e2e_ms, args.steps, world)
    # bytes crossing the bus per step: the planner-info blob in (the layout of
    # csrc/dp_layout.h: a 343-word header, 2 words per class, its
    # selectivities, 9 words per class member, then 16-byte aligned the
    # per-relation class masks (rows of whole 4-word groups), 2 pair
    # selectivities per class (rounded up to 4 words) and the plain-class
    # mask, plus the 3 n^2 tree tables of a tree-shaped graph; staged in
    # 512-word buckets); out, one copy of the engine's control block: 33 level
    # counters (24 B), the pair counter, the barrier words, the tree size, 64
    # plan nodes (28 B)
    q0 = qs[0]
    n_ec = len(q0.eq_classes)
    n_sels = sum(len(e.sels) for e in q0.eq_classes)
    n_fks = sum(len(e.members) for e in q0.eq_classes)
    ec_stride = (((n_ec + 31) // 32) + 3) // 4 * 4
    words = (343 + 2 * n_ec + n_sels + 9 * n_fks + 3) // 4 * 4
    words += N_RELS * ec_stride + (2 * n_ec + 3) // 4 * 4 + ec_stride + 3 * N_RELS * N_RELS
    h2d = 4 * ((words + 511) // 512 * 512)
    d2h = 33 * 24 + 8 + 16 + 4 + 4 + 64 * 28

    if rank == 0:
        peak, peak_kind = measured_peaks()
        alg_bytes = pairs * 32 + csgs * 20
        per_launch_bytes = alg_bytes / max(1, eval_launches)
        per_launch_s = (eval_ms / 1000.0) / max(1, eval_launches)
        achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
        traffic = profiled_figure("dram_bytes_per_launch")
        line = {
            "metric": METRIC, "value": value, "unit": "ms/query", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "b200",
            "config": {"workload": WORKLOAD, "seeds": SEEDS, "queries_per_step_per_gpu": 1,
                       "l2": "flushed before every step (256 MB write)", "parallelism": f"query-sharded x{world}",
                       "autotuned": {k: tuning[k] for k in ("single_narrow_level_sets", "single_wide_level_sets",
                                                            "batch_single_sets", "tune_ms")}},
            "evaluated_pairs_per_step": pairs / args.steps,
            "connected_sets_per_step": csgs / args.steps,
            "pairs_per_s": pairs / (tot_ms / 1000.0) if tot_ms > 0 else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_dp_tree (MPDP, persistent)", "eval_kernel_share": eval_ms / tot_ms if tot_ms else None,
                         "traffic_source": "profiles/k_dp_tree_snowflake25_traffic.txt (ncu of this benchmark's "
                                           "workload, mean of the timed launches)",
                         "l2_throughput_pct_of_peak": profiled_figure("l2_throughput_pct_of_peak"),
                         "issue_active_pct": profiled_figure("issue_active_pct")},
            "e2e": {"value": e2e_value, "unit": "ms/query", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": kernels,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_batched:
            line["batched"] = batched_section()
        if world == 1 and not args.no_served:
            line["served"] = served_section()
        if world == 1 and not args.no_configs:
            line["configs"] = configs_section(cpu=not args.no_cpu_baseline)
        if world == 1 and not args.no_cpu_baseline:
            med, mean, cores, ns = cpu_reference_sample(qs, capi.GPUQO_CPU_DPSUB_BICC_PARALLEL)
            line["cpu_baseline"] = {"value": med, "unit": "ms/query", "cores": cores, "kind": "reference",
                                    "mean": mean, "cpu_model": cpu_model(),
                                    "sample": f"median of {ns} snowflake-25 MPDP queries after one warm-up, "
                                              f"parallel_cpu_dpsub_bicc, {cores} threads, chunk 256"}
            ok, why = native_reference_usable()
            if ok:
                med_n, mean_n, _, nn = cpu_reference_sample(qs, capi.GPUQO_CPU_DPSUB_BICC_PARALLEL, native=True)
                line["cpu_baseline"]["march_native"] = {"value": med_n, "mean": mean_n, "runs": nn}
            else:
                line["cpu_baseline"]["march_native"] = {"skipped": why}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
