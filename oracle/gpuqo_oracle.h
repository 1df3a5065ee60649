/*
 * gpuqo_oracle.h - plain-C restatement of the reference's CPU join-order DP
 * (cpu_dpsub and cpu_dpsub_bicc), used ONLY as a test oracle.
 *
 * TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load libgpuqo_oracle.so.  The product library does not
 * link it, and nothing in the product path calls it.
 *
 * The ABI structs are the reference's (src/include/optimizer/gpuqo_common.h,
 * gpuqo_planner_info.h), so the same GpuqoPlannerInfoC bytes feed the
 * reference library, this oracle and the product.
 */
#ifndef GPUQO_ORACLE_H
#define GPUQO_ORACLE_H

#include <stdbool.h>
#include <stdint.h>

typedef uint64_t bitmapword;

typedef struct Bitmapset {
    int nwords;
    bitmapword words[];
} Bitmapset;

typedef struct PathCost { float startup; float total; } PathCost;
typedef struct GpuqoIndexInfo { bool available; bool unique; float rows; PathCost cost; } GpuqoIndexInfo;
typedef struct VarStats { float stadistinct; float stanullfrac; float mcvfreq; } VarStats;
typedef struct VarInfo { VarStats stats; GpuqoIndexInfo index; } VarInfo;

typedef struct EqClassInfo {
    void *eclass;
    Bitmapset *relids;
    float *sels;
    VarInfo *vars;
    Bitmapset **fk;
    struct EqClassInfo *next;
} EqClassInfo;

typedef struct BaseRelationC {
    Bitmapset *id;
    float rows;
    float tuples;
    PathCost cost;
    int width;
} BaseRelationC;

typedef struct GpuqoPlannerInfoC {
    int n_rels;
    BaseRelationC *base_rels;
    Bitmapset **edge_table;
    EqClassInfo *eq_classes;
    int n_eq_classes;
    int n_eq_class_sels;
    int n_eq_class_fks;
    int n_eq_class_vars;
} GpuqoPlannerInfoC;

typedef struct QueryTreeC {
    Bitmapset *id;
    float rows;
    PathCost cost;
    int width;
    struct QueryTreeC *left;
    struct QueryTreeC *right;
} QueryTreeC;

/* Same entry point and algorithm numbering as the reference
 * (gpuqo_main_internal.cu:177; gpuqo_common.h:13-29).  Supported here:
 * 3 = GPUQO_CPU_DPSUB, 5 = GPUQO_CPU_DPSUB_BICC.  Other values return NULL. */
QueryTreeC *gpuqo_run(int gpuqo_algorithm, GpuqoPlannerInfoC *info);
void oracle_free_query_tree(QueryTreeC *qt);

/* Plans of at least this many relations use the hash memo over the connected
 * sets (always from 29 relations on; up to 63).  Lower it to run small plans
 * through that driver too. */
extern int oracle_sparse_from_rels;


/* One make_join_relation evaluation on the caller's (unrelabelled) info. */
void oracle_eval_join(GpuqoPlannerInfoC *info, uint64_t left_id, uint64_t right_id,
                      const float *vals_in, float *vals_out);

#endif
