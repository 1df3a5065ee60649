/*
 * gpuqo_b200.h - C ABI of libgpuqo_b200.so, the B200 (sm_100a) join-order
 * dynamic programming library (DPsub / MPDP, IDP2 / UnionDP on top).
 *
 * Drop-in boundary.  The library replaces the reference's gpuqo object set
 * (the gpuqo_*.cu files under src/backend/optimizer/gpuqo, linked into postgres per
 * src/backend/Makefile:55-59) behind the same entry point and the same GUC
 * variables; the planner glue gpuqo_main.c (the caller) is unchanged.
 *
 * Struct layouts are the reference's, byte for byte, so a backend compiled
 * against src/include/optimizer/gpuqo_planner_info.h can call this library.
 * When those headers are already included, the declarations below are skipped.
 * tests/test_abi_reference.py compiles this header and the reference's headers
 * side by side and compares every size, offset and enum value.
 */
#ifndef GPUQO_B200_H
#define GPUQO_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Reference ABI types                                                     */
/* ---------------------------------------------------------------------- */
#if !defined(GPUQO_PLANNER_INFO_H) && !defined(GPUQO_COMMON_H)

/* Postgres nodes/bitmapset.h; re-declared by the reference in
 * src/backend/optimizer/gpuqo/gpuqo_postgres.cuh:29-33 */
#ifndef BITMAPSET_H
typedef uint64_t bitmapword;
typedef struct Bitmapset {
    int nwords;
    bitmapword words[];
} Bitmapset;
#endif

/* src/include/optimizer/gpuqo_common.h:13-29 */
typedef enum GpuqoAlgorithm {
    GPUQO_DPSIZE = 0,
    GPUQO_DPSUB,
    GPUQO_CPU_DPSIZE,
    GPUQO_CPU_DPSUB,
    GPUQO_CPU_DPSUB_PARALLEL,
    GPUQO_CPU_DPSUB_BICC,
    GPUQO_CPU_DPSUB_BICC_PARALLEL,
    GPUQO_CPU_DPCCP,
    GPUQO_DPE_DPSIZE,
    GPUQO_DPE_DPSUB,
    GPUQO_DPE_DPCCP,
    GPUQO_CPU_GOO,
    GPUQO_CPU_IKKBZ,
    GPUQO_CPU_LINEARIZED_DP,
    GPUQO_CPU_DPLIN
} GpuqoAlgorithm;

/* gpuqo_common.h:31-36 */
typedef enum GpuqoIDPType {
    GPUQO_IDP1 = 0,
    GPUQO_IDP2,
    GPUQO_UNION
} GpuqoIDPType;

/* gpuqo_common.h:91-113 */
typedef struct PathCost { float startup; float total; } PathCost;
typedef struct GpuqoIndexInfo { bool available; bool unique; float rows; PathCost cost; } GpuqoIndexInfo;
typedef struct VarStats { float stadistinct; float stanullfrac; float mcvfreq; } VarStats;
typedef struct VarInfo { VarStats stats; GpuqoIndexInfo index; } VarInfo;

/* src/include/optimizer/gpuqo_planner_info.h:17-55 */
typedef Bitmapset *EdgeMask;
typedef Bitmapset *RelationID;

typedef struct EqClassInfo {
    void *eclass;                 /* EquivalenceClass*, unused here */
    RelationID relids;
    float *sels;                  /* size*(size-1)/2, eqClassIndex order */
    VarInfo *vars;                /* one per member */
    RelationID *fk;               /* one per member, may be NULL */
    struct EqClassInfo *next;
} EqClassInfo;

typedef struct BaseRelationC {
    RelationID id;
    float rows;
    float tuples;
    PathCost cost;
    int width;
} BaseRelationC;

typedef struct GpuqoPlannerInfoC {
    int n_rels;
    BaseRelationC *base_rels;
    EdgeMask *edge_table;
    EqClassInfo *eq_classes;
    int n_eq_classes;
    int n_eq_class_sels;
    int n_eq_class_fks;
    int n_eq_class_vars;
} GpuqoPlannerInfoC;

typedef struct QueryTreeC {
    RelationID id;
    float rows;
    PathCost cost;
    int width;
    struct QueryTreeC *left;
    struct QueryTreeC *right;
} QueryTreeC;

#endif /* reference headers not included */

/* ---------------------------------------------------------------------- */
/* Entry point                                                             */
/* ---------------------------------------------------------------------- */

/*
 * Replaces: extern QueryTreeC* gpuqo_run(int gpuqo_algorithm, GpuqoPlannerInfoC* info)
 *   src/include/optimizer/gpuqo.h:23, impl src/backend/optimizer/gpuqo/
 *   gpuqo_main_internal.cu:177-185; caller gpuqo_main.c:584.
 *
 * gpuqo_algorithm: GPUQO_DPSUB runs the GPU DP - MPDP (biconnected-block
 *   csg-cmp enumeration) when gpuqo_dpsub_bicc_enable is set, plain DPsub
 *   (all-subsets enumeration with CCC) otherwise.  The CPU algorithm codes
 *   (GPUQO_CPU_DPSUB, GPUQO_CPU_DPSUB_BICC and their parallel/DPE variants)
 *   return the same plans as the reference's CPU engines; they are served by
 *   the same GPU kernels (plain DPsub for *_DPSUB, MPDP for *_BICC*).
 *   GPUQO_DPSIZE, GPUQO_CPU_DPSIZE and GPUQO_DPE_DPSIZE return the plans of
 *   the reference's cpu_dpsize (up to 31 relations).  Other codes (DPccp,
 *   heuristics) are outside this library's scope and return NULL with a
 *   message, as the reference does for unsupported combinations
 *   (gpuqo_main_internal.cu:75-78).
 * Exact DP: up to 31 relations on a dense memo; DPsub and MPDP of 32 to 63
 *   relations on a sparse memo over the connected sets
 *   (gpuqo_b200_sparse_from_rels).
 * IDP: when 1 < gpuqo_idp_n_iters < n_rels, gpuqo_idp_type selects IDP2
 *   (gpuqo_idp.cu:260) or UnionDP (gpuqo_dpdp_union.cu:448) over the GPU DP;
 *   sub-problems of up to 63 relations.
 *
 * The input is borrowed.  The returned tree and every id Bitmapset are
 * palloc'd (inside Postgres: the caller's memory context; standalone: the
 * library's malloc-based palloc).  Returns NULL on error, after printing a
 * message to stderr; gpuqo_b200_last_error() returns the code.
 */
QueryTreeC *gpuqo_run(int gpuqo_algorithm, GpuqoPlannerInfoC *info);

/* ---------------------------------------------------------------------- */
/* GUC variables (bound by address from guc.c; reference definition sites) */
/* ---------------------------------------------------------------------- */
extern int gpuqo_algorithm;                          /* gpuqo_main.c:43 */
extern int gpuqo_scratchpad_size_mb;                 /* gpuqo_dpsize.cu:41 */
extern int gpuqo_max_memo_size_mb;                   /* gpuqo_dpsize.cu:42 */
extern int gpuqo_min_memo_size_mb;                   /* gpuqo_dpsize.cu:43 */
extern int gpuqo_n_parallel;                         /* gpuqo_dpsub_common.cu:45 */
extern bool gpuqo_dpsub_filter_enable;               /* gpuqo_dpsub_filtered.cu:44 */
extern int gpuqo_dpsub_filter_threshold;             /* :45 */
extern int gpuqo_dpsub_filter_cpu_enum_threshold;    /* :46 */
extern int gpuqo_dpsub_filter_keys_overprovisioning; /* :47 */
extern bool gpuqo_dpsub_ccc_enable;                  /* :50 */
extern bool gpuqo_dpsub_csg_enable;                  /* :53 */
extern int gpuqo_dpsub_csg_threshold;                /* :54 */
extern bool gpuqo_dpsub_tree_enable;                 /* :57 */
extern bool gpuqo_dpsub_bicc_enable;                 /* :60 */
extern int gpuqo_dpe_n_threads;                      /* gpuqo_cpu_dpe.cu:33 */
extern int gpuqo_dpe_pairs_per_depbuf;               /* gpuqo_cpu_dpe.cu:34 */
extern int gpuqo_cpu_dpsub_parallel_chunk_size;      /* gpuqo_cpu_dpsub_parallel.cu:30 */
extern bool gpuqo_spanning_tree_enable;              /* gpuqo_spanning_tree.cu:15 */
extern int gpuqo_idp_n_iters;                        /* gpuqo_idp.cu:14 */
extern int gpuqo_idp_type;                           /* gpuqo_idp.cu:15 */
extern int gpuqo_dplin_csg_threshold_lindp;          /* gpuqo_cpu_dplin.cu:27 */
extern int gpuqo_dplin_threshold_lindp;              /* gpuqo_cpu_dplin.cu:28 */
extern int gpuqo_dplin_threshold_idp;                /* gpuqo_cpu_dplin.cu:29 */

/* ---------------------------------------------------------------------- */
/* Library extensions (no counterpart in the reference)                    */
/* ---------------------------------------------------------------------- */

/* Status codes of the extension entry points. */
enum {
    GPUQO_B200_OK = 0,
    GPUQO_B200_ERR_ARGS = 1,        /* bad arguments / unsupported input */
    GPUQO_B200_ERR_CUDA = 2,        /* CUDA runtime error */
    GPUQO_B200_ERR_NOMEM = 3,       /* device memory budget exceeded */
    GPUQO_B200_ERR_TOO_LARGE = 4,   /* exact DP beyond the dense-memo limit */
    GPUQO_B200_ERR_UNSUPPORTED = 5, /* algorithm outside this library */
    GPUQO_B200_ERR_CANCELLED = 6    /* InterruptPending was set */
};

/* Code of the last failed call on this thread (GPUQO_B200_OK if none). */
int gpuqo_b200_last_error(void);

/* Frees a tree returned by gpuqo_run / the batch API with pfree. */
void gpuqo_b200_free_query_tree(QueryTreeC *qt);

/* Counters of the last exact-DP run (summed over IDP sub-problems). */
typedef struct GpuqoB200Stats {
    uint64_t connected_sets;      /* csgs evaluated (levels >= 2) */
    uint64_t evaluated_pairs;     /* valid csg-cmp pairs costed */
    uint64_t filtered_subsets;    /* candidate subsets unranked and tested */
    uint64_t memo_bytes;          /* device memo footprint */
    double   device_ms;           /* device time of the DP (CUDA events) */
    double   eval_kernel_ms;      /* summed time of the evaluate kernels */
    uint32_t eval_kernel_launches;
    uint32_t n_subproblems;       /* exact DP runs (1, or IDP iterations) */
    uint32_t kernel_launches;     /* kernels launched by the DP runs */
    uint32_t fallback_sets;       /* tree-mode sets re-evaluated in exact order (ties, NaN) */
    uint32_t barrier_timeouts;    /* persistent launches whose grid barrier gave up (rerun per level) */
    double   handoff_device_ms;   /* batch: device time of the queries large enough to run alone */
} GpuqoB200Stats;
void gpuqo_b200_get_stats(GpuqoB200Stats *out);

/* When non-zero, per-kernel CUDA events are recorded around every evaluate
 * launch (for the kernel-time figures in the stats); off by default. */
extern int gpuqo_b200_profile_kernels;

/* When non-zero (default), MPDP on a tree-shaped query graph runs as one
 * persistent cooperative kernel with a grid barrier between levels; zero
 * selects the per-level launches (also used automatically when a cooperative
 * launch is not possible or its barrier times out). */
extern int gpuqo_b200_persistent;

/* Every grid-barrier wait of the persistent kernels is bounded (4 s and 2^26
 * polls).  When one gives up, the kernel raises an error flag, every block
 * leaves, the host reruns that DP with per-level launches (same plan) and the
 * device's engines keep using per-level launches until
 * gpuqo_b200_reset_persistent() clears that state (it returns how many
 * engines it cleared).  gpuqo_b200_barrier_poll_limit, when > 0, replaces the
 * 2^26 polls: a small value makes waits run out on purpose, to exercise that
 * path without a fault; 0 (default) keeps the built-in limits. */
extern int gpuqo_b200_barrier_poll_limit;
int gpuqo_b200_reset_persistent(void);

/* Device-memory budget of the exact-DP arenas in MB (0, the default: no
 * limit but the device's).  A DP whose dense memo, level lists or batch wave
 * would need more is refused before anything is allocated: the call returns
 * NULL (or the status) with GPUQO_B200_ERR_NOMEM and the library's state is
 * unchanged, so later calls that fit succeed.  A failed cudaMalloc is
 * reported the same way. */
extern int gpuqo_b200_device_memory_mb;

/* Exact DPs (DPsub, MPDP) over at least this many relations use the sparse
 * memo: the connected sets are enumerated on the host, an open-addressing
 * table on the device maps each set to its memo slot, and one launch per
 * level evaluates every set with 64-bit relation sets.  Default 32, the end of
 * the dense memo (one entry per subset of up to 31 relations); the sparse memo
 * reaches 63 relations when the graph has at most 2^25 connected sets and no
 * set more than 2^26 candidate splits.  A lower value sends smaller queries
 * the same way (their plans are the dense memo's, bit for bit); 0 or a value
 * above 63 keeps the default. */
extern int gpuqo_b200_sparse_from_rels;

/* Connected sets the host lists for a sparse-memo DP of a graph that is not
 * a tree before it hands the listing to the device (level by level, the
 * device table deduplicating; the arrays are then sized for the sparse memo's
 * whole capacity).  0 (default): 65536.  Trees are always listed on the
 * device.  Plans do not depend on it. */
extern int gpuqo_b200_sparse_host_list;

/*
 * Device-resident timing of the exact DP of one query (< 32 relations, no
 * IDP): the planner info is converted and uploaded once, then the captured DP
 * graph is replayed warmup + iters times; CUDA events on the library's stream
 * time each replay, with a 256 MB L2 flush between replays when flush_l2 is
 * set.  *ms_per_iter receives the mean device milliseconds per replay and
 * *tree (if non-NULL) the plan of the last replay.  Returns a status code.
 */
int gpuqo_b200_time_resident(int gpuqo_algorithm, GpuqoPlannerInfoC *info, int warmup, int iters,
                             int flush_l2, double *ms_per_iter, QueryTreeC **tree);

/*
 * One node of a plan returned in caller-provided storage: relids in the
 * caller's numbering (relation i is bit i+1), children as indices into the
 * same array (-1 for leaves), node 0 is the root.
 */
typedef struct GpuqoB200PlanNode {
    uint64_t relids;
    int32_t left, right;
    float rows;
    float startup;
    float total;
    int32_t width;
} GpuqoB200PlanNode;

/*
 * No counterpart in the reference.  Exact DP (same algorithm selection and
 * same plans as gpuqo_run) that allocates nothing, for callers that cannot
 * allocate device memory: a Postgres backend that must not leak GPU memory
 * when elog(ERROR) longjmps out of a cancelled query, or a process whose
 * device memory is owned by another pool.  All scratch lives in one static
 * device array of about 6.7 MB that every GPU loading this library keeps
 * until exit; queries are limited to 18 relations and to a device planner
 * info of 6144 32-bit words (about 270 two-member equivalence classes, more
 * than the 153 edges of an 18-relation clique); larger ones return
 * GPUQO_B200_ERR_TOO_LARGE with a message naming the limit.  The caller passes the planner
 * info (host, as for gpuqo_run), a CUDA stream (cudaStream_t, NULL for the
 * default stream) and an output array of at least 2*n_rels-1 nodes; the call
 * returns after the stream work completes.  The first call on each device
 * looks up the scratch address (cudaGetSymbolAddress) - make it before any
 * stream capture.  Calls share the scratch: calls that overlap on the GPU
 * race.  Returns a status code.
 */
int gpuqo_b200_run_noalloc(int gpuqo_algorithm, const GpuqoPlannerInfoC *info, void *cuda_stream,
                           GpuqoB200PlanNode *nodes, int max_nodes, int *n_nodes);

/*
 * Batched exact DP: optimises n_queries independent queries in one call.
 * MPDP queries of up to 30 relations (no IDP) are packed into waves whose
 * dense memos share one device arena of at most gpuqo_b200_batch_memory_mb;
 * each wave runs level by level with one enumeration and one evaluation
 * launch per level for all of its queries.  Other queries (plain DPsub, IDP,
 * very large biconnected blocks) run one by one through gpuqo_run's path.
 * Trees are written to out[i] (palloc'd, NULL on error); every plan is the
 * one gpuqo_run returns for that query.  Returns a status code.
 */
extern int gpuqo_b200_batch_memory_mb;
int gpuqo_b200_run_batch(int gpuqo_algorithm, GpuqoPlannerInfoC **infos,
                         int n_queries, QueryTreeC **out);

/*
 * Devices of the batch entry and of the planner service (no reference
 * counterpart): 1 (the default) uses the calling thread's current device;
 * N > 1 the N devices from the current one on, wrapping around the visible
 * ones; 0 every visible device.  Queries are independent, so a batch is
 * split by estimated work (gpuqo_b200_plan_shards) and each device runs its
 * share with its own engines on its own host thread; the service gives each
 * request to the device with the fewest requests in flight.  No data crosses
 * between devices.  Plans do not depend on the setting.
 */
extern int gpuqo_b200_devices;

/* The split used by the batch: item i of weight work[i] goes to device
 * device_of_item[i] in [0, n_devices), longest first onto the least-loaded
 * device (lower index first on ties).  A pure host function. */
int gpuqo_b200_plan_shards(const double *work, int n_items, int n_devices, int *device_of_item);

/*
 * Continuous-batching planner service (standalone planning processes; inside
 * a Postgres backend use gpuqo_run).  Requests are planned concurrently, at
 * most max_inflight at a time (later ones wait for a slot); every exact DP a
 * request needs (one, or one per IDP2 / UnionDP iteration) is run by a single
 * scheduler in level-synchronous waves together with the pending sub-problems
 * of all other requests, each wave admitted by dense-memo bytes
 * (wave_memory_mb).  A request's plan equals gpuqo_run's for the same query
 * and the GUC settings current at submit time (gpuqo_algorithm argument,
 * gpuqo_dpsub_bicc_enable, gpuqo_idp_n_iters, gpuqo_idp_type).
 *
 * submit copies what it needs from info (the caller may free it on return)
 * and returns a ticket; wait blocks until that request is planned and hands
 * back its tree (palloc'd) and its latency from submit to completion.
 */
typedef struct GpuqoB200ServerStats {
    uint64_t completed;             /* requests planned */
    uint64_t waves;                 /* batched waves run */
    uint64_t batched_subproblems;   /* exact DPs run inside waves */
    uint64_t single_subproblems;    /* exact DPs run one by one */
    double device_ms;               /* device time of all waves and singles */
    double busy_ms;                 /* wall time the scheduler spent running waves and singles */
    double starved_ms;              /* wall time the scheduler waited for sub-problems while requests were open */
} GpuqoB200ServerStats;

/*
 * Autotuner (no reference counterpart).  Kernel variants and the hand-off
 * between batch waves and single launches are chosen by connected-set count;
 * gpuqo_b200_autotune measures the three crossovers on the current device (about
 * a second, synthetic star queries of 14 to 24 relations) and installs them for
 * later calls.  Plans never depend on these choices.  Until it runs,
 * gpuqo_b200_get_tuning reports the built-in defaults (tuned = 0).
 */
typedef struct GpuqoB200Tuning {
    double single_narrow_level_sets; /* tree queries with up to this many connected sets per relation
                                        (their total over n) run the 2-blocks-per-SM kernel */
    double single_wide_level_sets;   /* tree queries with more connected sets per relation than this run
                                        the 4-blocks-per-SM kernel; the 3-blocks one in between */
    double batch_single_sets;  /* batches run tree queries above this many connected sets as single launches */
    double tune_ms;            /* wall time of the last gpuqo_b200_autotune, 0 if it never ran */
    int tuned;
} GpuqoB200Tuning;

int gpuqo_b200_autotune(GpuqoB200Tuning *out);
int gpuqo_b200_get_tuning(GpuqoB200Tuning *out);
/* Installs the three crossovers of *in for the current device without
 * measuring (for a process that restores the result of an earlier
 * gpuqo_b200_autotune on the same kind of device, or pins a kernel variant
 * for profiling); tune_ms is ignored, tuned is stored as given.  Negative or
 * NaN crossovers: GPUQO_B200_ERR_ARGS. */
int gpuqo_b200_set_tuning(const GpuqoB200Tuning *in);

/* Batching window of the planner service's schedulers, in microseconds
 * (default 100): when sub-problems are pending but some of the lane's running
 * planners are between two sub-problems, the scheduler waits up to this long
 * for them before it starts the wave (a wave costs about the same device time
 * for a few sub-problems as for many).  0 starts every wave at once.  Plans
 * do not depend on it. */
extern int gpuqo_b200_server_batch_window_us;

int gpuqo_b200_server_start(int max_inflight, int wave_memory_mb);
int gpuqo_b200_server_submit(int gpuqo_algorithm, GpuqoPlannerInfoC *info, uint64_t *ticket);
int gpuqo_b200_server_wait(uint64_t ticket, QueryTreeC **out, double *latency_ms);
/* Cancels one request: it stops before its next exact DP (IDP iterations
 * included) and its wait returns GPUQO_B200_ERR_CANCELLED, unless it had
 * already finished; the other requests are unaffected.  Unknown ticket:
 * GPUQO_B200_ERR_ARGS.  (InterruptPending still cancels every request.) */
int gpuqo_b200_server_cancel(uint64_t ticket);
int gpuqo_b200_server_stats(GpuqoB200ServerStats *out);
int gpuqo_b200_server_stop(void);

#ifdef __cplusplus
}
#endif

#endif /* GPUQO_B200_H */
