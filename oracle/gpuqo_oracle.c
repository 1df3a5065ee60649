/*
 * gpuqo_oracle.c - plain-C restatement of the reference's sequential CPU
 * join-order DP, as a TEST ORACLE.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as a checker.  The product never links it.
 *
 * Parity pin: this restatement is checked against the reference's own code
 * compiled from its sources (oracle/_ref/libgpuqo_ref.so, oracle/Makefile)
 * and against the golden fixtures in tests/golden/ generated from it.
 *
 * What it restates (file:line in the reference tree,
 * src/backend/optimizer/gpuqo/):
 *   gpuqo_run dispatch ......... gpuqo_main_internal.cu:82-185
 *   C -> internal conversion ... gpuqo_planner_info.cu:134-200, setParams :114-131
 *   BFS relabelling ............ gpuqo_bfs_indexing.cu:14-55,
 *                                gpuqo_remapper.cu:34-300 (remap info / tree)
 *   row estimation ............. gpuqo_row_estimation.cuh:26-160
 *   cost model ................. gpuqo_cost.cuh:46-157,
 *                                gpuqo_cost_postgres.cuh:86-862
 *   connectivity ............... gpuqo_filter.cuh:119-160
 *   cpu_dpsub .................. gpuqo_cpu_dpsub.cuh:26-40,
 *                                gpuqo_cpu_dpsub.cu:32-78,
 *                                gpuqo_cpu_common.cuh:169-211,
 *                                gpuqo_cpu_sequential.cu:63-132
 *   cpu_dpsub_bicc ............. gpuqo_cpu_dpsub_bicc.cu:46-236
 *
 * Floating point: every expression keeps the reference's operand order and
 * types (float, except the double division in fkselc_of_ec); the file is
 * built with -ffp-contract=off so no multiply-add is fused.  Conversions of
 * out-of-range floats to int follow x86-64 cvttss2si (result INT_MIN), which
 * is what the reference's host build does.
 *
 * Memo: dense, indexed by (relid mask >> 1), instead of the reference's
 * std::unordered_map, up to 28 relations; lookups are equivalent (a set is
 * present iff it was inserted).  From 29 to 63 relations (or from
 * oracle_sparse_from_rels on) a hash memo over the connected sets only, same
 * visiting order and candidates (run_dp_sparse).
 */
#include "gpuqo_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* GUCs read by the restated path (same names as the reference)             */
/* ------------------------------------------------------------------------ */
double seq_page_cost = 1.0;
double random_page_cost = 4.0;
double cpu_tuple_cost = 0.01;
double cpu_index_tuple_cost = 0.005;
double cpu_operator_cost = 0.0025;
int effective_cache_size = 524288;
double disable_cost = 1.0e10;
bool enable_seqscan = true;
bool enable_indexscan = true;
bool enable_tidscan = false;
bool enable_sort = true;
bool enable_hashagg = true;
bool enable_nestloop = true;
bool enable_mergejoin = false;
bool enable_hashjoin = true;
int work_mem = 4096;
int gpuqo_idp_n_iters = 0;
int gpuqo_idp_type = 1;

#define MAXN 64
#define ORACLE_MAX_DENSE 28

typedef uint64_t mask_t;

typedef struct {
    float effective_cache_size, seq_page_cost, random_page_cost, cpu_tuple_cost,
        cpu_index_tuple_cost, cpu_operator_cost, disable_cost;
    bool enable_seqscan, enable_indexscan, enable_tidscan, enable_sort,
        enable_hashagg, enable_nestloop, enable_mergejoin, enable_hashjoin;
    int work_mem;
} Params;

typedef struct {
    mask_t id;
    float rows, tuples;
    int width;
    PathCost cost;
    bool composite;
} BaseRel;

typedef struct {
    int n_rels;
    Params p;
    BaseRel base[MAXN];
    mask_t edge[MAXN];
    int n_ec;
    mask_t *ec_relids;   /* n_ec */
    float *ec_sels;      /* sum s(s-1)/2 */
    mask_t *ec_fks;      /* sum s */
    VarInfo *ec_vars;    /* sum s */
} Info;

typedef struct {
    float rows;
    PathCost cost;
    int width;
} Rel;

typedef struct Tree {
    mask_t id;
    float rows;
    PathCost cost;
    int width;
    struct Tree *left, *right;
} Tree;

/* ------------------------------------------------------------------------ */
/* bit helpers (gpuqo_bitmapset.cuh:49-190)                                  */
/* ------------------------------------------------------------------------ */
static inline int popc(mask_t x) { return __builtin_popcountll(x); }
static inline mask_t lowest(mask_t x) { return x & (~x + 1); }
static inline int lowest_pos(mask_t x) { return __builtin_ffsll((long long)x) - 1; }
static inline mask_t all_lower(mask_t x) { return lowest(x) - 1; }
static inline mask_t nth(int n) { return (mask_t)1 << n; }
/* gpuqo_bitmapset.cuh:302-305 */
static inline mask_t next_subset(mask_t subset, mask_t set) { return set & (subset - set); }
static inline mask_t pdep(mask_t val, mask_t mask) {
    mask_t r = 0;
    for (mask_t bb = 1; mask; bb += bb) {
        mask_t low = mask & (~mask + 1);
        if (val & bb) r |= low;
        mask &= mask - 1;
    }
    return r;
}

/* gpuqo_common.h:72-79 */
static inline int eq_class_n_sels(int s) { return s * (s - 1) / 2; }
static inline int eq_class_index(int l, int r, int size) {
    if (l > r) { int t = l; l = r; r = t; }
    return l * size - l * (l + 1) / 2 + (r - l - 1);
}

/* float -> int as x86-64 cvttss2si: truncation, INT_MIN when out of range. */
static inline int f2i_x86(float f) {
    if (!(f > -2147483649.0f && f < 2147483648.0f)) return INT_MIN;
    return (int)f;
}

static inline int clz64(uint64_t x) { return __builtin_clzll(x); }
/* gpuqo_cost_postgres.cuh:86-99 */
static inline int floor_log2(long num) { return (int)(sizeof(num) * 8) - 1 - clz64((uint64_t)num); }
static inline int ceil_log2(long num) {
    int res = floor_log2(num);
    if ((1L << res) == num) return res;
    return res + 1;
}

/* ------------------------------------------------------------------------ */
/* connectivity (gpuqo_filter.cuh:119-160)                                   */
/* ------------------------------------------------------------------------ */
static mask_t grow(mask_t from, mask_t subset, const mask_t *edge) {
    mask_t V = 0, N = from;
    while (N) {
        int idx = lowest_pos(N) - 1;
        V |= nth(idx + 1);
        N |= edge[idx];
        N &= subset;
        N &= ~V;
    }
    return V;
}

static bool is_connected(mask_t relid, const mask_t *edge) {
    if (!relid) return false;
    return grow(lowest(relid), relid, edge) == relid;
}

/* ------------------------------------------------------------------------ */
/* row estimation (gpuqo_row_estimation.cuh)                                 */
/* ------------------------------------------------------------------------ */
/* :26-45 */
static float fkselc_of_ec(const Info *info, int off_fk, mask_t ec, mask_t outer_rels, mask_t inner_rels) {
    mask_t tmp = outer_rels;
    while (tmp) {
        mask_t out_id = lowest(tmp);
        int out_idx = popc(all_lower(out_id) & ec);
        mask_t match = inner_rels & info->ec_fks[off_fk + out_idx];
        if (match) {
            int in_idx = lowest_pos(match) - 1;
            return (float)(1.0 / (double)fmaxf(1.0f, info->base[in_idx].tuples));
        }
        tmp &= ~out_id;
    }
    return NAN;
}

/* :49-88 */
static float estimate_ec_selectivity(const Info *info, mask_t ec, int off_sels, int off_fks,
                                     mask_t l, mask_t r) {
    int size = popc(ec);
    mask_t ml = ec & l, mr = ec & r;
    if (!ml || !mr) return 1.0f;
    float fk = fkselc_of_ec(info, off_fks, ec, ml, mr);
    if (!isnan(fk)) return fk;
    fk = fkselc_of_ec(info, off_fks, ec, mr, ml);
    if (!isnan(fk)) return fk;
    int il = popc(all_lower(ml) & ec);
    int ir = popc(all_lower(mr) & ec);
    return info->ec_sels[off_sels + eq_class_index(il, ir, size)];
}

/* :93-118 */
static float estimate_join_selectivity(const Info *info, mask_t l, mask_t r) {
    float sel = 1.0f;
    int off_sels = 0, off_fks = 0;
    for (int i = 0; i < info->n_ec; i++) {
        mask_t ec = info->ec_relids[i];
        sel *= estimate_ec_selectivity(info, ec, off_sels, off_fks, l, r);
        int s = popc(ec);
        off_sels += eq_class_n_sels(s);
        off_fks += s;
    }
    return sel;
}

/* :123-132 */
static float estimate_join_rows(const Info *info, mask_t lid, const Rel *l, mask_t rid, const Rel *r) {
    float sel = estimate_join_selectivity(info, lid, rid);
    float rows = sel * l->rows * r->rows;
    return rows > 1 ? roundf(rows) : 1;
}

/* ------------------------------------------------------------------------ */
/* cost model (gpuqo_cost_postgres.cuh, gpuqo_cost.cuh)                      */
/* ------------------------------------------------------------------------ */
typedef struct { int n_quals; float startup, per_tuple; } QualCost;
typedef struct { float mcvfreq, bucketsize; } BucketStats;
typedef struct { int numbuckets, numbatches, num_skew_mcvs; } HtszRes;
typedef struct { bool inner_unique, indexed_join_quals; float joinrows, outer_match_frac, match_count; } CostExtra;

/* :850-862 */
static float clamp_row_est(float nrows) {
    if (nrows <= 1.0f) nrows = 1.0f;
    else nrows = rintf(nrows);
    return nrows;
}

#define MAXALIGN8(LEN) (((uintptr_t)(LEN) + 7) & ~((uintptr_t)7))
/* :820-841 */
static float relation_byte_size(float tuples, int width) {
    return tuples * (float)(MAXALIGN8(width) + 24);
}
static float page_size(float tuples, int width) {
    return ceilf(relation_byte_size(tuples, width) / (float)8192);
}

/* :790-812 */
static QualCost cost_qual_eval(const Info *info, mask_t l, mask_t r) {
    QualCost c = {0, 0.0f, 0.0f};
    for (int i = 0; i < info->n_ec; i++) {
        mask_t ec = info->ec_relids[i];
        if (!(ec & l) || !(ec & r)) continue;
        c.per_tuple += info->p.cpu_operator_cost;
        c.n_quals++;
    }
    return c;
}

/* :480-621 */
static HtszRes exec_choose_hash_table_size(float ntuples, int tupwidth, int work_mem_kb) {
    HtszRes res;
    res.numbatches = 1;
    if (ntuples <= 0.0f) ntuples = 1000.0f;
    int tupsize = 32 + (int)MAXALIGN8(tupwidth);
    float inner_rel_bytes = ntuples * tupsize;
    long hash_table_bytes = work_mem_kb * 1024L;
    float space_allowed = hash_table_bytes;
    long skew_table_bytes = hash_table_bytes * 2 / 100;
    res.num_skew_mcvs = (int)(skew_table_bytes / (tupsize + 84));
    if (res.num_skew_mcvs > 0) hash_table_bytes -= skew_table_bytes;
    long max_pointers = (long)(space_allowed / (float)sizeof(void *));
    {
        unsigned long a = (unsigned long)max_pointers, b = (unsigned long)(0x3fffffffUL / sizeof(void *));
        max_pointers = (long)(a < b ? a : b);
    }
    long mppow2 = 1L << ceil_log2(max_pointers);
    if (max_pointers != mppow2) max_pointers = mppow2 / 2;
    if (max_pointers > (long)INT_MAX / 2) max_pointers = (long)INT_MAX / 2;
    float dbuckets = ceilf(ntuples / 1);
    dbuckets = fminf(dbuckets, (float)max_pointers);
    res.numbuckets = (int)dbuckets;
    if (res.numbuckets < 1024) res.numbuckets = 1024;
    res.numbuckets = 1 << ceil_log2(res.numbuckets);
    long bucket_bytes = (long)(sizeof(void *) * (unsigned long)res.numbuckets);
    if (inner_rel_bytes + (float)bucket_bytes > (float)hash_table_bytes) {
        long bucket_size = (long)(tupsize * 1 + sizeof(void *));
        long lbuckets = 1L << ceil_log2(hash_table_bytes / bucket_size);
        if (lbuckets > max_pointers) lbuckets = max_pointers;
        res.numbuckets = (int)lbuckets;
        res.numbuckets = 1 << ceil_log2(res.numbuckets);
        bucket_bytes = (long)(res.numbuckets * sizeof(void *));
        float dbatch = ceilf(inner_rel_bytes / (float)(hash_table_bytes - bucket_bytes));
        dbatch = fminf(dbatch, (float)max_pointers);
        int minbatch = (int)dbatch;
        int p2 = 1 << ceil_log2(minbatch);
        res.numbatches = p2 > 2 ? p2 : 2;
    }
    return res;
}

/* :705-787 */
static float estimate_hash_bucketsize_one(const VarInfo *v, const BaseRel *baserel, int nbuckets) {
    float estfract, ndistinct, mcvfreq, avgfreq;
    ndistinct = v->stats.stadistinct;
    if (ndistinct < 0.0f) ndistinct = -ndistinct * baserel->tuples;
    if (ndistinct <= 0.0f) return 0.1f;
    avgfreq = (1.0f - v->stats.stanullfrac) / ndistinct;
    if (baserel->tuples > 0.0f) {
        ndistinct *= baserel->rows / baserel->tuples;
        ndistinct = clamp_row_est(ndistinct);
    }
    if (ndistinct > (float)nbuckets) estfract = 1.0f / (float)nbuckets;
    else estfract = 1.0f / ndistinct;
    mcvfreq = v->stats.mcvfreq;
    if (avgfreq > 0.0f && mcvfreq > avgfreq) estfract *= mcvfreq / avgfreq;
    if (estfract < 1.0e-6f) estfract = 1.0e-6f;
    else if (estfract > 1.0f) estfract = 1.0f;
    return estfract;
}

/* :624-679 */
static BucketStats estimate_hash_bucket_stats(const Info *info, mask_t outer, mask_t inner, int nbuckets) {
    BucketStats st;
    st.bucketsize = 1.0f;
    st.mcvfreq = 1.0f;
    int off_vars = 0;
    for (int i = 0; i < info->n_ec; off_vars += popc(info->ec_relids[i]), i++) {
        mask_t ec = info->ec_relids[i];
        mask_t ml = ec & outer, mr = ec & inner;
        if (!ml || !mr) continue;
        while (mr) {
            mask_t in_id = lowest(mr);
            int in_idx = popc(all_lower(in_id) & ec);
            const BaseRel *baserel = &info->base[lowest_pos(in_id) - 1];
            const VarInfo *v = &info->ec_vars[off_vars + in_idx];
            float this_bs = estimate_hash_bucketsize_one(v, baserel, nbuckets);
            if (st.bucketsize > this_bs) st.bucketsize = this_bs;
            if (st.mcvfreq > v->stats.mcvfreq) st.mcvfreq = v->stats.mcvfreq;
            mr &= ~in_id;
        }
    }
    return st;
}

/* :114-279 */
static PathCost cost_nestloop(const Info *info, mask_t outer_id, const Rel *outer,
                              mask_t inner_id, const Rel *inner, const CostExtra *extra) {
    float startup_cost = 0.0f, run_cost = 0.0f, cpu_per_tuple, inner_run_cost, inner_rescan_run_cost;
    float outer_path_rows = outer->rows, inner_path_rows = inner->rows, ntuples;
    if (!info->p.enable_nestloop) startup_cost += info->p.disable_cost;
    startup_cost += inner->cost.startup + outer->cost.startup;
    run_cost += outer->cost.total - outer->cost.startup;
    if (outer_path_rows > 1.0f) run_cost += (outer_path_rows - 1.0f) * inner->cost.startup;
    inner_run_cost = inner->cost.total - inner->cost.startup;
    inner_rescan_run_cost = inner_run_cost;
    if (extra->inner_unique) {
        float outer_matched_rows, outer_unmatched_rows, inner_scan_frac;
        outer_matched_rows = rintf(outer_path_rows * extra->outer_match_frac);
        outer_unmatched_rows = outer_path_rows - outer_matched_rows;
        inner_scan_frac = 2.0f / (extra->match_count + 1.0f);
        ntuples = outer_matched_rows * inner_path_rows * inner_scan_frac;
        if (extra->indexed_join_quals) {
            run_cost += inner_run_cost * inner_scan_frac;
            if (outer_matched_rows > 1.0f)
                run_cost += (outer_matched_rows - 1.0f) * inner_rescan_run_cost * inner_scan_frac;
            run_cost += outer_unmatched_rows * inner_rescan_run_cost / inner_path_rows;
        } else {
            ntuples += outer_unmatched_rows * inner_path_rows;
            run_cost += inner_run_cost;
            if (outer_unmatched_rows >= 1.0f) outer_unmatched_rows -= 1.0f;
            else outer_matched_rows -= 1.0f;
            if (outer_matched_rows > 0.0f)
                run_cost += outer_matched_rows * inner_rescan_run_cost * inner_scan_frac;
            if (outer_unmatched_rows > 0.0f)
                run_cost += outer_unmatched_rows * inner_rescan_run_cost;
        }
    } else {
        run_cost += inner_run_cost;
        if (outer_path_rows > 1.0f) run_cost += (outer_path_rows - 1.0f) * inner_rescan_run_cost;
        ntuples = outer_path_rows * inner_path_rows;
    }
    QualCost rq = cost_qual_eval(info, inner_id, outer_id);
    startup_cost += rq.startup;
    cpu_per_tuple = info->p.cpu_tuple_cost + rq.per_tuple;
    run_cost += cpu_per_tuple * ntuples;
    PathCost pc = {startup_cost, startup_cost + run_cost};
    return pc;
}

/* :291-468 */
static PathCost cost_hashjoin(const Info *info, mask_t outer_id, const Rel *outer,
                              mask_t inner_id, const Rel *inner, CostExtra extra) {
    float startup_cost = 0.0f, run_cost = 0.0f, cpu_per_tuple, hashjointuples, virtualbuckets;
    float outer_path_rows = outer->rows, inner_path_rows = inner->rows;
    float inner_path_rows_total = inner_path_rows;
    if (!info->p.enable_hashjoin) startup_cost += info->p.disable_cost;
    QualCost hq = cost_qual_eval(info, outer_id, inner_id);
    startup_cost += outer->cost.startup;
    run_cost += outer->cost.total - outer->cost.startup;
    startup_cost += inner->cost.total;
    startup_cost += (info->p.cpu_operator_cost * hq.n_quals + info->p.cpu_tuple_cost) * inner_path_rows;
    run_cost += info->p.cpu_operator_cost * hq.n_quals * outer_path_rows;
    HtszRes h = exec_choose_hash_table_size(inner_path_rows_total, inner->width, info->p.work_mem);
    if (h.numbatches > 1) {
        float outerpages = page_size(outer_path_rows, outer->width);
        float innerpages = page_size(inner_path_rows, inner->width);
        startup_cost += info->p.seq_page_cost * innerpages;
        run_cost += info->p.seq_page_cost * (innerpages + 2.0f * outerpages);
    }
    virtualbuckets = (float)h.numbuckets * (float)h.numbatches;
    BucketStats bs = estimate_hash_bucket_stats(info, outer_id, inner_id, f2i_x86(virtualbuckets));
    if (relation_byte_size(clamp_row_est(inner_path_rows * bs.mcvfreq), inner->width) >
        (float)(info->p.work_mem * 1024L))
        startup_cost += info->p.disable_cost;
    if (extra.inner_unique) {
        float outer_matched_rows = rintf(outer_path_rows * extra.outer_match_frac);
        float inner_scan_frac = 2.0f / (extra.match_count + 1.0f);
        startup_cost += hq.startup;
        run_cost += hq.per_tuple * outer_matched_rows *
                    clamp_row_est(inner_path_rows * bs.bucketsize * inner_scan_frac) * 0.5f;
        run_cost += hq.per_tuple * (outer_path_rows - outer_matched_rows) *
                    clamp_row_est(inner_path_rows / virtualbuckets) * 0.05f;
        hashjointuples = outer_matched_rows;
    } else {
        startup_cost += hq.startup;
        run_cost += hq.per_tuple * outer_path_rows *
                    clamp_row_est(inner_path_rows * bs.bucketsize) * 0.5f;
        hashjointuples = extra.joinrows;
    }
    cpu_per_tuple = info->p.cpu_tuple_cost;
    run_cost += cpu_per_tuple * hashjointuples;
    PathCost pc = {startup_cost, startup_cost + run_cost};
    return pc;
}

/* gpuqo_cost.cuh:46-73 */
static bool is_inner_unique(const Info *info, mask_t outer_id, mask_t inner_id) {
    if (popc(inner_id) != 1) return false;
    int off_vars = 0;
    for (int i = 0; i < info->n_ec; off_vars += popc(info->ec_relids[i]), i++) {
        mask_t ec = info->ec_relids[i];
        mask_t ml = ec & outer_id, mr = ec & inner_id;
        if (!ml || !mr) continue;
        mask_t in_id = lowest(mr);
        int in_idx = popc(all_lower(in_id) & ec);
        const VarInfo *v = &info->ec_vars[off_vars + in_idx];
        if (v->index.available && v->index.unique) return true;
    }
    return false;
}

/* gpuqo_cost.cuh:81-157 */
static PathCost calc_join_cost(const Info *info, mask_t outer_id, const Rel *outer,
                               mask_t inner_id, const Rel *inner, float join_rel_rows) {
    PathCost min_cost, tmp;
    CostExtra extra;
    extra.inner_unique = is_inner_unique(info, outer_id, inner_id);
    extra.indexed_join_quals = false;
    extra.joinrows = join_rel_rows;
    extra.outer_match_frac = join_rel_rows / (outer->rows * inner->rows);
    extra.match_count = inner->rows;
    min_cost.startup = 0.0f;
    min_cost.total = NAN;
    tmp = cost_nestloop(info, outer_id, outer, inner_id, inner, &extra);
    if (isnan(min_cost.total) || tmp.total < min_cost.total) min_cost = tmp;
    if (info->p.enable_hashjoin) {
        tmp = cost_hashjoin(info, outer_id, outer, inner_id, inner, extra);
        if (tmp.total < min_cost.total) min_cost = tmp;
    }
    extra.indexed_join_quals = true;
    if (popc(inner_id) == 1) {
        const BaseRel *baserel = &info->base[lowest_pos(inner_id) - 1];
        if (!baserel->composite) {
            int off_vars = 0;
            for (int i = 0; i < info->n_ec; off_vars += popc(info->ec_relids[i]), i++) {
                mask_t ec = info->ec_relids[i];
                mask_t ml = ec & outer_id, mr = ec & inner_id;
                if (!ml || !mr) continue;
                mask_t in_id = lowest(mr);
                int in_idx = popc(all_lower(in_id) & ec);
                const VarInfo *v = &info->ec_vars[off_vars + in_idx];
                if (!v->index.available) continue;
                Rel idx_inner;
                idx_inner.rows = v->index.rows;
                idx_inner.cost = v->index.cost;
                idx_inner.width = 0;
                tmp = cost_nestloop(info, outer_id, outer, inner_id, &idx_inner, &extra);
                if (tmp.total < min_cost.total) min_cost = tmp;
            }
        }
    }
    return min_cost;
}

/* ------------------------------------------------------------------------ */
/* dense memo + DP drivers                                                   */
/* ------------------------------------------------------------------------ */
typedef struct {
    Rel rel;
    mask_t left, right;
    bool present;
} MemoEntry;

typedef struct {
    const Info *info;
    MemoEntry *memo;   /* indexed by mask >> 1 */
} Dp;

/* gpuqo_cpu_common.cuh:169-211 (make_join_relation + do_join, strict '<') */
static void join_into(const Info *info, MemoEntry *je, mask_t left_id, const MemoEntry *le, mask_t right_id,
                      const MemoEntry *re) {
    Rel jr;
    jr.rows = estimate_join_rows(info, left_id, &le->rel, right_id, &re->rel);
    jr.cost = calc_join_cost(info, left_id, &le->rel, right_id, &re->rel, jr.rows);
    jr.width = le->rel.width + re->rel.width;
    if (je->present) {
        if (jr.cost.total < je->rel.cost.total) {
            je->rel = jr;
            je->left = left_id;
            je->right = right_id;
        }
    } else {
        je->present = true;
        je->rel = jr;
        je->left = left_id;
        je->right = right_id;
    }
}

static void dp_join(Dp *dp, mask_t left_id, mask_t right_id) {
    join_into(dp->info, &dp->memo[(left_id | right_id) >> 1], left_id, &dp->memo[left_id >> 1], right_id,
              &dp->memo[right_id >> 1]);
}

/* gpuqo_cpu_dpsub.cu:32-78 */
static void dpsub_enumerate_subsets(Dp *dp, mask_t join_id) {
    mask_t left_id = lowest(join_id);
    while (left_id != join_id) {
        mask_t right_id = join_id & ~left_id;
        if (left_id && right_id) {
            if (dp->memo[left_id >> 1].present && dp->memo[right_id >> 1].present)
                dp_join(dp, left_id, right_id);
        }
        left_id = next_subset(left_id, join_id);
    }
}

/* gpuqo_cpu_dpsub_bicc.cu:65-170 (iterative Hopcroft-Tarjan, same DFS and
 * output order) */
typedef struct { int u; mask_t edges; bool remain; } CallEl;
typedef struct { int u, v; } EdgeEl;

static int find_blocks(const Info *info, mask_t set, mask_t *blocks) {
    CallEl call[4 * MAXN * MAXN];
    EdgeEl estack[2 * MAXN * MAXN];
    int ctop = 0, etop = 0, nb = 0;
    bool visited[MAXN + 1];
    int depth[MAXN + 1], low[MAXN + 1];
    int parent[MAXN + 1];
    for (int i = 0; i <= MAXN; i++) { visited[i] = false; depth[i] = -1; parent[i] = 0; low[i] = INT_MAX; }
    call[ctop++] = (CallEl){lowest_pos(set), 0, false};
    int curr_depth = 1;
    while (ctop > 0) {
        CallEl el = call[--ctop];
        if (!el.edges) {
            visited[el.u] = true;
            depth[el.u] = curr_depth++;
            mask_t edges = info->edge[el.u - 1] & set;
            if (edges) call[ctop++] = (CallEl){el.u, edges, false};
        } else {
            int v = lowest_pos(el.edges);
            if (el.remain) {
                if (low[v] >= depth[el.u]) {
                    mask_t block = 0;
                    EdgeEl e;
                    do {
                        e = estack[--etop];
                        block |= nth(e.u) | nth(e.v);
                    } while (e.u != el.u || e.v != v);
                    blocks[nb++] = block;
                }
                if (low[v] < low[el.u]) low[el.u] = low[v];
                el.edges &= ~nth(v);
                if (el.edges) call[ctop++] = (CallEl){el.u, el.edges, false};
            } else {
                if (!visited[v]) {
                    estack[etop++] = (EdgeEl){el.u, v};
                    parent[v] = el.u;
                    call[ctop++] = (CallEl){el.u, el.edges, true};
                    call[ctop++] = (CallEl){v, 0, false};
                } else if (parent[el.u] != v && depth[v] < depth[el.u]) {
                    estack[etop++] = (EdgeEl){el.u, v};
                    if (depth[v] < low[el.u]) low[el.u] = depth[v];
                    el.edges &= ~nth(v);
                    if (el.edges) call[ctop++] = (CallEl){el.u, el.edges, false};
                } else {
                    el.edges &= ~nth(v);
                    if (el.edges) call[ctop++] = (CallEl){el.u, el.edges, false};
                }
            }
        }
    }
    return nb;
}

/* gpuqo_cpu_dpsub_bicc.cu:172-236 */
static void bicc_enumerate_subsets(Dp *dp, mask_t set) {
    mask_t blocks[MAXN * 2];
    int nb = find_blocks(dp->info, set, blocks);
    for (int b = 0; b < nb; b++) {
        mask_t block = blocks[b];
        mask_t lb = lowest(block);
        while (lb != block) {
            mask_t rb = block & ~lb;
            mask_t left_id = grow(lowest(lb), set & ~rb, dp->info->edge);
            mask_t right_id = grow(lowest(rb), set & ~lb, dp->info->edge);
            if ((left_id | right_id) == set) dp_join(dp, left_id, right_id);
            lb = next_subset(lb, block);
        }
    }
}

static Tree *build_tree(const Dp *dp, mask_t id) {
    const MemoEntry *e = &dp->memo[id >> 1];
    if (!e->present) return NULL;
    Tree *t = (Tree *)calloc(1, sizeof(Tree));
    t->id = id;
    t->rows = e->rel.rows;
    t->cost = e->rel.cost;
    t->width = e->rel.width;
    if (popc(id) > 1) {
        t->left = build_tree(dp, e->left);
        t->right = build_tree(dp, e->right);
    }
    return t;
}

/* gpuqo_cpu_sequential.cu:63-132 + gpuqo_cpu_dpsub.cuh:26-40 (non-IDP order) */
static Tree *run_dp(const Info *info, bool bicc) {
    int n = info->n_rels;
    if (n > ORACLE_MAX_DENSE) {
        fprintf(stderr, "gpuqo_oracle: n=%d exceeds the dense-memo limit %d\n", n, ORACLE_MAX_DENSE);
        return NULL;
    }
    Dp dp;
    dp.info = info;
    dp.memo = (MemoEntry *)calloc((size_t)1 << n, sizeof(MemoEntry));
    if (!dp.memo) return NULL;
    for (int i = 0; i < n; i++) {
        MemoEntry *e = &dp.memo[info->base[i].id >> 1];
        e->present = true;
        e->rel.rows = info->base[i].rows;
        e->rel.cost = info->base[i].cost;
        e->rel.width = info->base[i].width;
        e->left = e->right = 0;
    }
    for (mask_t i = 1; i < nth(n); i++) {
        mask_t join_id = i << 1;
        if (!is_connected(join_id, info->edge)) continue;
        if (bicc) bicc_enumerate_subsets(&dp, join_id);
        else dpsub_enumerate_subsets(&dp, join_id);
    }
    mask_t final_id = 0;
    for (int i = 0; i < n; i++) final_id |= info->base[i].id;
    Tree *t = build_tree(&dp, final_id);
    free(dp.memo);
    return t;
}

/* ------------------------------------------------------------------------ */
/* sparse memo: the same DP over the connected sets only (29 to 63 relations) */
/* ------------------------------------------------------------------------ */
/*
 * The reference's memo is a std::unordered_map (gpuqo_cpu_sequential.cu:63)
 * holding only the sets that were joined, and its non-IDP enumeration visits
 * every subset in increasing integer order but skips those that are not
 * connected (gpuqo_cpu_dpsub.cuh:26-40).  This driver visits exactly the
 * connected sets, in the same increasing integer order, with a hash memo; the
 * candidates of each set are the reference's, in the reference's order:
 *   DPsub: every L of S, ascending (gpuqo_cpu_dpsub.cu:35-75), joined when
 *          both L and S - L are present, i.e. connected; here the connected
 *          subsets of S are listed and sorted, which is the same sequence;
 *   MPDP:  per block of S in find_blocks order, every lb of the block
 *          ascending, grown on both sides, joined when the sides cover S
 *          (gpuqo_cpu_dpsub_bicc.cu:180-232).  For a block that is a simple
 *          cycle of m >= 4 relations only the m(m - 1) arcs can cover S (a
 *          non-contiguous lb grows to the part hanging off one of its arcs),
 *          so the arcs are taken in ascending order and the other lb, which
 *          join nothing, are skipped.  A block of more than 26 relations that
 *          is not a cycle is refused (2^26 candidates per set).
 * Bound: at most 2^24 connected sets.
 */
int oracle_sparse_from_rels = ORACLE_MAX_DENSE + 1;

#define SPARSE_MAX_SETS (1u << 24)
#define SPARSE_MAX_BLOCK 26

typedef struct {
    mask_t *keys;      /* 0 = empty slot (no set is empty) */
    uint32_t *val;
    uint32_t cap;      /* power of two */
    uint32_t count;
} SetMap;

static uint32_t setmap_slot(mask_t k, uint32_t cap) {
    return (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> 40) & (cap - 1u);
}

static bool setmap_init(SetMap *m, uint32_t want) {
    m->cap = 16;
    while (m->cap < 2u * want) m->cap <<= 1;
    m->count = 0;
    m->keys = (mask_t *)calloc(m->cap, sizeof(mask_t));
    m->val = (uint32_t *)calloc(m->cap, sizeof(uint32_t));
    return m->keys && m->val;
}

static void setmap_free(SetMap *m) {
    free(m->keys);
    free(m->val);
}

static long setmap_get(const SetMap *m, mask_t k) {
    for (uint32_t i = setmap_slot(k, m->cap);; i = (i + 1u) & (m->cap - 1u)) {
        if (m->keys[i] == k) return (long)m->val[i];
        if (m->keys[i] == 0) return -1;
    }
}

/* insert if absent; returns false when it was present (or on no memory) */
static bool setmap_add(SetMap *m, mask_t k, uint32_t v) {
    if (2u * (m->count + 1u) > m->cap) {
        SetMap g;
        g.cap = m->cap * 2u;
        g.count = 0;
        g.keys = (mask_t *)calloc(g.cap, sizeof(mask_t));
        g.val = (uint32_t *)calloc(g.cap, sizeof(uint32_t));
        if (!g.keys || !g.val) {
            setmap_free(&g);
            return false;
        }
        for (uint32_t i = 0; i < m->cap; i++)
            if (m->keys[i]) setmap_add(&g, m->keys[i], m->val[i]);
        setmap_free(m);
        *m = g;
    }
    uint32_t i = setmap_slot(k, m->cap);
    for (; m->keys[i]; i = (i + 1u) & (m->cap - 1u))
        if (m->keys[i] == k) return false;
    m->keys[i] = k;
    m->val[i] = v;
    m->count++;
    return true;
}

typedef struct {
    mask_t *v;
    uint32_t n, cap;
} MaskList;

static bool masklist_push(MaskList *l, mask_t x) {
    if (l->n == l->cap) {
        uint32_t c = l->cap ? 2u * l->cap : 64u;
        mask_t *nv = (mask_t *)realloc(l->v, (size_t)c * sizeof(mask_t));
        if (!nv) return false;
        l->v = nv;
        l->cap = c;
    }
    l->v[l->n++] = x;
    return true;
}

static int cmp_mask(const void *a, const void *b) {
    const mask_t x = *(const mask_t *)a, y = *(const mask_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* the connected subsets of `within` (all of them when within is every
 * relation), by extension with one neighbour at a time; false past `limit` */
static bool connected_subsets(const Info *info, mask_t within, uint32_t limit, MaskList *out) {
    SetMap seen;
    if (!setmap_init(&seen, 64)) return false;
    bool ok = true;
    for (mask_t x = within; x && ok; x &= x - 1) {
        ok = masklist_push(out, lowest(x)) && setmap_add(&seen, lowest(x), 0);
    }
    uint32_t lvl_start = 0;
    while (ok && lvl_start < out->n) {
        const uint32_t lvl_end = out->n;
        for (uint32_t i = lvl_start; i < lvl_end && ok; i++) {
            const mask_t S = out->v[i];
            mask_t nb = 0;
            for (mask_t x = S; x; x &= x - 1) nb |= info->edge[lowest_pos(x) - 1];
            nb &= within & ~S;
            for (; nb && ok; nb &= nb - 1) {
                const mask_t T = S | lowest(nb);
                if (setmap_get(&seen, T) >= 0) continue;
                if (out->n >= limit) {
                    ok = false;
                    break;
                }
                ok = setmap_add(&seen, T, 0) && masklist_push(out, T);
            }
        }
        lvl_start = lvl_end;
    }
    setmap_free(&seen);
    return ok;
}

typedef struct {
    const Info *info;
    SetMap index;       /* set -> entry */
    MemoEntry *memo;    /* in ascending set order */
} SparseDp;

static MemoEntry *sparse_entry(const SparseDp *dp, mask_t id) {
    const long i = setmap_get(&dp->index, id);
    return i < 0 ? NULL : &dp->memo[i];
}

static void sparse_join(SparseDp *dp, MemoEntry *je, mask_t left_id, mask_t right_id) {
    const MemoEntry *le = sparse_entry(dp, left_id), *re = sparse_entry(dp, right_id);
    if (le && re && le->present && re->present) join_into(dp->info, je, left_id, le, right_id, re);
}

static bool is_simple_cycle(const Info *info, mask_t block) {
    if (popc(block) < 4) return false;
    for (mask_t x = block; x; x &= x - 1)
        if (popc(info->edge[lowest_pos(x) - 1] & block) != 2) return false;
    return true;
}

/* MPDP candidates of one set (see above); false for an oversized block */
static bool sparse_bicc_set(SparseDp *dp, MemoEntry *je, mask_t set) {
    const Info *info = dp->info;
    mask_t blocks[MAXN * 2];
    const int nb = find_blocks(info, set, blocks);
    for (int b = 0; b < nb; b++) {
        const mask_t block = blocks[b];
        const int m = popc(block);
        if (is_simple_cycle(info, block)) {
            /* walk the cycle from its lowest relation; arcs are contiguous runs */
            mask_t order[MAXN];
            int v = lowest_pos(block), prev = -1;
            for (int i = 0; i < m; i++) {
                order[i] = nth(v);
                const mask_t nbrs = info->edge[v - 1] & block & ~(prev >= 0 ? nth(prev) : 0);
                prev = v;
                v = lowest_pos(nbrs);
            }
            mask_t arcs[MAXN * MAXN];
            int na = 0;
            for (int st = 0; st < m; st++) {
                mask_t a = 0;
                for (int len = 1; len < m; len++) {
                    a |= order[(st + len - 1) % m];
                    arcs[na++] = a;
                }
            }
            qsort(arcs, (size_t)na, sizeof(mask_t), cmp_mask);
            for (int i = 0; i < na; i++) {
                const mask_t lb = arcs[i], rb = block & ~lb;
                const mask_t left_id = grow(lowest(lb), set & ~rb, info->edge);
                const mask_t right_id = grow(lowest(rb), set & ~lb, info->edge);
                if ((left_id | right_id) == set) sparse_join(dp, je, left_id, right_id);
            }
            continue;
        }
        if (m > SPARSE_MAX_BLOCK) {
            fprintf(stderr, "gpuqo_oracle: a block of %d relations exceeds the sparse driver\n", m);
            return false;
        }
        mask_t lb = lowest(block);
        while (lb != block) {
            const mask_t rb = block & ~lb;
            const mask_t left_id = grow(lowest(lb), set & ~rb, info->edge);
            const mask_t right_id = grow(lowest(rb), set & ~lb, info->edge);
            if ((left_id | right_id) == set) sparse_join(dp, je, left_id, right_id);
            lb = next_subset(lb, block);
        }
    }
    return true;
}

/* DPsub candidates of one set: its connected subsets, ascending */
static bool sparse_dpsub_set(SparseDp *dp, MemoEntry *je, mask_t set) {
    MaskList subs = {0};
    if (!connected_subsets(dp->info, set, SPARSE_MAX_SETS, &subs)) {
        free(subs.v);
        return false;
    }
    qsort(subs.v, subs.n, sizeof(mask_t), cmp_mask);
    for (uint32_t i = 0; i < subs.n; i++) {
        const mask_t left_id = subs.v[i];
        if (left_id == set) continue;
        sparse_join(dp, je, left_id, set & ~left_id);
    }
    free(subs.v);
    return true;
}

static Tree *build_tree_sparse(const SparseDp *dp, mask_t id) {
    const MemoEntry *e = sparse_entry(dp, id);
    if (!e || !e->present) return NULL;
    Tree *t = (Tree *)calloc(1, sizeof(Tree));
    t->id = id;
    t->rows = e->rel.rows;
    t->cost = e->rel.cost;
    t->width = e->rel.width;
    if (popc(id) > 1) {
        t->left = build_tree_sparse(dp, e->left);
        t->right = build_tree_sparse(dp, e->right);
    }
    return t;
}

static Tree *run_dp_sparse(const Info *info, bool bicc) {
    const int n = info->n_rels;
    mask_t full = 0;
    for (int i = 0; i < n; i++) full |= info->base[i].id;
    MaskList sets = {0};
    if (!connected_subsets(info, full, SPARSE_MAX_SETS, &sets)) {
        fprintf(stderr, "gpuqo_oracle: more than %u connected sets\n", SPARSE_MAX_SETS);
        free(sets.v);
        return NULL;
    }
    qsort(sets.v, sets.n, sizeof(mask_t), cmp_mask);
    SparseDp dp;
    dp.info = info;
    dp.memo = (MemoEntry *)calloc(sets.n, sizeof(MemoEntry));
    Tree *t = NULL;
    bool ok = dp.memo && setmap_init(&dp.index, sets.n);
    for (uint32_t i = 0; ok && i < sets.n; i++) ok = setmap_add(&dp.index, sets.v[i], i);
    for (int i = 0; ok && i < n; i++) {
        MemoEntry *e = sparse_entry(&dp, info->base[i].id);
        e->present = true;
        e->rel.rows = info->base[i].rows;
        e->rel.cost = info->base[i].cost;
        e->rel.width = info->base[i].width;
        e->left = e->right = 0;
    }
    for (uint32_t i = 0; ok && i < sets.n; i++) {
        const mask_t set = sets.v[i];
        if (popc(set) < 2) continue;
        ok = bicc ? sparse_bicc_set(&dp, &dp.memo[i], set) : sparse_dpsub_set(&dp, &dp.memo[i], set);
    }
    if (ok) t = build_tree_sparse(&dp, full);
    if (dp.memo) setmap_free(&dp.index);
    free(dp.memo);
    free(sets.v);
    return t;
}

/* ------------------------------------------------------------------------ */
/* conversion, BFS remap and back                                            */
/* ------------------------------------------------------------------------ */
static mask_t bms_to_mask(const Bitmapset *b) {
    if (!b) return 0;
    return b->words[0];
}

static void free_info(Info *info) {
    free(info->ec_relids);
    free(info->ec_sels);
    free(info->ec_fks);
    free(info->ec_vars);
}

/* gpuqo_planner_info.cu:114-200 */
static void convert_info(const GpuqoPlannerInfoC *c, Info *info) {
    memset(info, 0, sizeof(*info));
    info->n_rels = c->n_rels;
    info->p.effective_cache_size = effective_cache_size;
    info->p.random_page_cost = random_page_cost;
    info->p.seq_page_cost = seq_page_cost;
    info->p.cpu_tuple_cost = cpu_tuple_cost;
    info->p.cpu_index_tuple_cost = cpu_index_tuple_cost;
    info->p.cpu_operator_cost = cpu_operator_cost;
    info->p.disable_cost = disable_cost;
    info->p.enable_seqscan = enable_seqscan;
    info->p.enable_indexscan = enable_indexscan;
    info->p.enable_tidscan = enable_tidscan;
    info->p.enable_sort = enable_sort;
    info->p.enable_hashagg = enable_hashagg;
    info->p.enable_nestloop = enable_nestloop;
    info->p.enable_mergejoin = enable_mergejoin;
    info->p.enable_hashjoin = enable_hashjoin;
    info->p.work_mem = work_mem;
    for (int i = 0; i < c->n_rels; i++) {
        info->edge[i] = bms_to_mask(c->edge_table[i]);
        info->base[i].id = bms_to_mask(c->base_rels[i].id);
        info->base[i].rows = c->base_rels[i].rows;
        info->base[i].tuples = c->base_rels[i].tuples;
        info->base[i].width = c->base_rels[i].width;
        info->base[i].cost = c->base_rels[i].cost;
        info->base[i].composite = false;
    }
    info->n_ec = c->n_eq_classes;
    info->ec_relids = (mask_t *)calloc(c->n_eq_classes + 1, sizeof(mask_t));
    info->ec_sels = (float *)calloc(c->n_eq_class_sels + 1, sizeof(float));
    info->ec_fks = (mask_t *)calloc(c->n_eq_class_fks + 1, sizeof(mask_t));
    info->ec_vars = (VarInfo *)calloc(c->n_eq_class_vars + 1, sizeof(VarInfo));
    int i = 0, off_sels = 0, off_fks = 0;
    for (const EqClassInfo *ec = c->eq_classes; ec != NULL; ec = ec->next, i++) {
        info->ec_relids[i] = bms_to_mask(ec->relids);
        int s = popc(info->ec_relids[i]);
        int ns = eq_class_n_sels(s);
        for (int j = 0; j < ns; j++) info->ec_sels[off_sels + j] = ec->sels[j];
        for (int j = 0; j < s; j++) {
            info->ec_fks[off_fks + j] = bms_to_mask(ec->fk[j]);
            info->ec_vars[off_fks + j] = ec->vars[j];
        }
        off_sels += ns;
        off_fks += s;
    }
}

/* gpuqo_bfs_indexing.cu:14-55: to_of_from[from_idx] = to_idx */
static int bfs_order(const Info *info, int *from_of_to) {
    int queue[MAXN];
    int front = 0, back = 0, bfs_idx = 0;
    queue[back++] = 0;
    mask_t seen = nth(1);
    while (front != back && bfs_idx < info->n_rels) {
        int b = queue[front++];
        mask_t edges = info->edge[b];
        from_of_to[bfs_idx++] = b;
        while (edges) {
            int next = lowest_pos(edges);
            if (!(seen & nth(next))) queue[back++] = next - 1;
            edges &= ~nth(next);
        }
        seen |= info->edge[b];
    }
    return bfs_idx;
}

/* gpuqo_remapper.cu:34-277 for a relabelling of single relations */
static void remap_info(const Info *from, Info *to, const int *from_of_to, int n_to) {
    int to_of_from[MAXN];
    for (int i = 0; i < MAXN; i++) to_of_from[i] = -1;
    for (int t = 0; t < n_to; t++) to_of_from[from_of_to[t]] = t;
    memset(to, 0, sizeof(*to));
    to->n_rels = n_to;
    to->p = from->p;
#define REMAP(m) ({ mask_t _m = (m), _o = 0; \
        for (int _t = 0; _t < n_to; _t++) if (_m & nth(from_of_to[_t] + 1)) _o |= nth(_t + 1); _o; })
    for (int t = 0; t < n_to; t++) {
        to->edge[t] = REMAP(from->edge[from_of_to[t]]) & ~nth(t + 1);
        const BaseRel *b = &from->base[from_of_to[t]];
        to->base[t] = *b;
        to->base[t].id = nth(t + 1);
    }
    int n_sels = 0, n_fks = 0;
    for (int i = 0; i < from->n_ec; i++) {
        int s = popc(from->ec_relids[i]);
        n_sels += eq_class_n_sels(s);
        n_fks += s;
    }
    to->n_ec = from->n_ec;
    to->ec_relids = (mask_t *)calloc(from->n_ec + 1, sizeof(mask_t));
    to->ec_sels = (float *)calloc(n_sels + 1, sizeof(float));
    to->ec_fks = (mask_t *)calloc(n_fks + 1, sizeof(mask_t));
    to->ec_vars = (VarInfo *)calloc(n_fks + 1, sizeof(VarInfo));
    int off_sels = 0, off_fks = 0;
    for (int i = 0; i < from->n_ec; i++) {
        mask_t ecf = from->ec_relids[i];
        mask_t ect = REMAP(ecf);
        int s = popc(ecf);
        to->ec_relids[i] = ect;
        for (int lt = 0; lt < s; lt++) {
            mask_t id_lt = pdep(nth(lt), ect);
            mask_t id_lf = nth(from_of_to[lowest_pos(id_lt) - 1] + 1);
            int lf = popc(all_lower(id_lf) & ecf);
            for (int rt = lt + 1; rt < s; rt++) {
                mask_t id_rt = pdep(nth(rt), ect);
                mask_t id_rf = nth(from_of_to[lowest_pos(id_rt) - 1] + 1);
                int rf = popc(all_lower(id_rf) & ecf);
                to->ec_sels[off_sels + eq_class_index(lt, rt, s)] =
                    from->ec_sels[off_sels + eq_class_index(lf, rf, s)];
            }
            to->ec_fks[off_fks + lt] = REMAP(from->ec_fks[off_fks + lf]);
            to->ec_vars[off_fks + lt] = from->ec_vars[off_fks + lf];
        }
        off_sels += eq_class_n_sels(s);
        off_fks += s;
    }
#undef REMAP
}

static Bitmapset *mask_to_bms(mask_t m) {
    Bitmapset *b = (Bitmapset *)calloc(1, sizeof(Bitmapset) + sizeof(bitmapword));
    b->nwords = 1;
    b->words[0] = m;
    return b;
}

/* gpuqo_remapper.cu:279-300 + gpuqo_planner_info.cu:256-270 */
static QueryTreeC *tree_to_c(const Tree *t, const int *from_of_to, int n_to) {
    if (!t) return NULL;
    QueryTreeC *q = (QueryTreeC *)calloc(1, sizeof(QueryTreeC));
    mask_t orig = 0;
    for (int k = 0; k < n_to; k++)
        if (t->id & nth(k + 1)) orig |= nth(from_of_to[k] + 1);
    q->id = mask_to_bms(orig);
    q->left = tree_to_c(t->left, from_of_to, n_to);
    q->right = tree_to_c(t->right, from_of_to, n_to);
    q->width = t->width;
    q->cost = t->cost;
    q->rows = t->rows;
    return q;
}

static void free_tree(Tree *t) {
    if (!t) return;
    free_tree(t->left);
    free_tree(t->right);
    free(t);
}

void oracle_free_query_tree(QueryTreeC *qt) {
    if (!qt) return;
    oracle_free_query_tree(qt->left);
    oracle_free_query_tree(qt->right);
    free(qt->id);
    free(qt);
}

QueryTreeC *gpuqo_run(int gpuqo_algorithm, GpuqoPlannerInfoC *info_c) {
    if (gpuqo_algorithm != 3 && gpuqo_algorithm != 5) return NULL;
    if (info_c->n_rels > MAXN - 1 || info_c->n_rels < 1) return NULL;
    Info info, remapped;
    convert_info(info_c, &info);
    int from_of_to[MAXN];
    int n_to = bfs_order(&info, from_of_to);
    remap_info(&info, &remapped, from_of_to, n_to);
    const bool sparse = n_to > ORACLE_MAX_DENSE || (oracle_sparse_from_rels > 0 && n_to >= oracle_sparse_from_rels);
    Tree *t = sparse ? run_dp_sparse(&remapped, gpuqo_algorithm == 5) : run_dp(&remapped, gpuqo_algorithm == 5);
    QueryTreeC *res = tree_to_c(t, from_of_to, n_to);
    free_tree(t);
    free_info(&remapped);
    free_info(&info);
    return res;
}

/*
 * Single join evaluation on the caller's (unrelabelled) planner info, for
 * arithmetic-consistency checks of plans too large for a full oracle run:
 * given the children's (rows, startup, total, width), returns the join's, as
 * make_join_relation computes it (gpuqo_cpu_common.cuh:169-186).
 * vals_in: [l_rows, l_startup, l_total, l_width, r_rows, r_startup, r_total,
 * r_width]; vals_out: [rows, startup, total, width].
 */
void oracle_eval_join(GpuqoPlannerInfoC *info_c, uint64_t left_id, uint64_t right_id,
                      const float *vals_in, float *vals_out) {
    if (info_c->n_rels < 1 || info_c->n_rels > MAXN - 1) {
        for (int i = 0; i < 4; i++) vals_out[i] = NAN;
        return;
    }
    Info info;
    convert_info(info_c, &info);
    Rel l, r;
    l.rows = vals_in[0]; l.cost.startup = vals_in[1]; l.cost.total = vals_in[2]; l.width = (int)vals_in[3];
    r.rows = vals_in[4]; r.cost.startup = vals_in[5]; r.cost.total = vals_in[6]; r.width = (int)vals_in[7];
    float rows = estimate_join_rows(&info, left_id, &l, right_id, &r);
    PathCost c = calc_join_cost(&info, left_id, &l, right_id, &r, rows);
    vals_out[0] = rows;
    vals_out[1] = c.startup;
    vals_out[2] = c.total;
    vals_out[3] = (float)(l.width + r.width);
    free_info(&info);
}
