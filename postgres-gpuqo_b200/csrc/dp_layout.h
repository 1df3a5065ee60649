// dp_layout.h - layout of the device planner-info blob, shared by the host
// code that builds it and the kernels that read it.
#pragma once

#include <cmath>
#include <cstdint>

#ifndef __CUDACC__
#define GQB_HD
#else
#define GQB_HD __host__ __device__
#endif

namespace gqb {

constexpr int kMaxRels = 32;      // compact masks are 32-bit
constexpr int kWarp = 32;

// ---------------------------------------------------------------------------
// Device planner info blob (built on the host, copied into shared memory by
// every CTA).  Layout: DevHeader, then
//   uint32 ec_relids[n_ec]; uint32 ec_off[n_ec] (off_sels << 16 | off_fks);
//   float sels[n_sels]; uint32 fks[n_fks]; DevVar vars[n_fks]
// ---------------------------------------------------------------------------
// A class member's variable.  The bucket-size terms depend only on the
// variable's statistics and its base relation's rows and tuples, so they are
// computed once on the host (devvar_bucket_terms) instead of per join pair.
struct DevVar {
    float bs_nd;                          // ndistinct scaled to the relation's rows and clamped
    float bs_inv_nd;                      // 1 / bs_nd
    float bs_mcv_ratio;                   // mcvfreq / avgfreq (applies when flags bit3)
    float mcvfreq;
    float idx_rows, idx_startup, idx_total;
    uint32_t flags;                       // bit0 index.available, bit1 index.unique,
                                          // bit2 no ndistinct (estimate 0.1), bit3 mcv ratio applies
};
static_assert(sizeof(DevVar) == 32, "DevVar layout");

constexpr uint32_t kVarNoDistinct = 4u;
constexpr uint32_t kVarMcvRatio = 8u;

// The relation-only part of __estimate_hash_bucketsize
// (gpuqo_cost_postgres.cuh:705-787): every operation below is the
// reference's, in its order, in IEEE single precision (built without
// contraction on the host), so the terms equal those the device would
// compute per pair.
GQB_HD inline void devvar_bucket_terms(DevVar &v, float stadistinct, float stanullfrac, float mcvfreq,
                                       float rel_rows, float rel_tuples) {
    float ndistinct = stadistinct;
    v.flags &= ~(kVarNoDistinct | kVarMcvRatio);
    v.mcvfreq = mcvfreq;
    v.bs_nd = 0.0f;
    v.bs_inv_nd = 0.0f;
    v.bs_mcv_ratio = 0.0f;
    if (ndistinct < 0.0f) ndistinct = -ndistinct * rel_tuples;
    if (ndistinct <= 0.0f) {
        v.flags |= kVarNoDistinct;
        return;
    }
    const float avgfreq = (1.0f - stanullfrac) / ndistinct;
    if (rel_tuples > 0.0f) {
        ndistinct *= rel_rows / rel_tuples;
        ndistinct = ndistinct <= 1.0f ? 1.0f : rintf(ndistinct);   // clamp_row_est
    }
    v.bs_nd = ndistinct;
    v.bs_inv_nd = 1.0f / ndistinct;
    if (avgfreq > 0.0f && mcvfreq > avgfreq) {
        v.flags |= kVarMcvRatio;
        v.bs_mcv_ratio = mcvfreq / avgfreq;
    }
}

struct DevHeader {
    int n, n_ec, n_sels, n_fks;
    float cpu_operator_cost, cpu_tuple_cost, seq_page_cost, disable_cost;
    int work_mem, enable_nestloop, enable_hashjoin;
    uint32_t composite_mask;
    uint32_t blob_words;                  // total blob size in 32-bit words
    uint32_t max_block;                   // largest biconnected block of the query graph
    uint32_t tree_mode;                   // query graph is a tree (tree tables present)
    uint32_t ec_masked;                   // tree_mode and every class is a 2-member class on an edge
    uint32_t tree_tab;                    // word offset of the tree tables (see below), 0 if none
    // memo widths carry the inner hash table size (see memo_width_word): set
    // when every width is >= 0 and all of them sum to less than 2^21
    uint32_t hz_packed;
    // key index of a candidate in the block (MPDP) enumeration: 0 = the MPDP
    // index (block, subset of the block), 1 = the plain-DPsub index of the
    // same split (gpuqo_dpsub_csg_enable: DPsub's winner from its valid
    // pairs only, see dpsub_index)
    uint32_t index_order;
    uint32_t adj[kMaxRels];
    float rows[kMaxRels];
    float tuples[kMaxRels];
    float startup[kMaxRels];
    float total[kMaxRels];
    int width[kMaxRels];
    // fkselc_of_ec's value for a foreign key into relation i:
    // (float)(1.0 / (double)fmaxf(1.0f, tuples[i])) (gpuqo_row_estimation.cuh:36-38)
    float fksel[kMaxRels];
    // ec_masked: the classes on the edge between relation i and its parent
    // when the query tree is rooted at relation 0
    uint32_t edge_ec[kMaxRels];
    // ec_masked: ec_selectivity of two-member class i (members x < y) with x
    // on the outer side (edge_sel[0][i]) and with y there (edge_sel[1][i]);
    // gpuqo_row_estimation.cuh:49-88 returns a FK selectivity or the class's
    // stored selectivity, no arithmetic, so the host fills the table exactly
    float edge_sel[2][kMaxRels];
    // every class has exactly two members (DevInfoView::pair_sel then holds
    // the selectivity of every class in both orientations)
    uint32_t all_pairs;
    uint32_t pad_[3];
};

// Tree tables (tree_mode), appended after the class arrays: for every root r
// of the query tree and relation v, with children visited in increasing
// index order,
//   tab[0*n*n + r*n + v] = relations of v's subtree,
//   tab[1*n*n + r*n + v] = relations preceding v in preorder,
//   tab[2*n*n + r*n + v] = proper ancestors of v.
// A connected set S is a subtree; the reference's block search walks it from
// its lowest relation r in exactly this preorder.
GQB_HD inline uint32_t tree_tab_words(int n) { return 3u * (uint32_t)n * (uint32_t)n; }

struct DevInfoView {
    const DevHeader *h;
    const uint32_t *ec_relids;
    const uint32_t *ec_off;
    const float *sels;
    const uint32_t *fks;
    const DevVar *vars;
    // rel_ecs[v * ec_stride(n_ec) + w]: bit b set when class 32 w + b has
    // relation v as a member (ec_words(n_ec) words per relation, each row
    // padded to a multiple of 4 words and 16-byte aligned for vector loads)
    const uint32_t *rel_ecs;
    // pair_sel[2 i + o]: ec_selectivity of two-member class i (members x < y)
    // with x on the outer side (o = 0) or y there (o = 1); NaN for classes of
    // another size, which take the general path
    const float *pair_sel;
    // plain[w] bit b: class 32 w + b has two members whose variables carry no
    // statistics and no index (ndistinct unknown, MCV frequency 0): as the
    // inner side of a join such a class always contributes the bucket-size
    // estimate 0.1, the MCV frequency 0 and no unique index (ec_stride words)
    const uint32_t *plain;
};

GQB_HD inline int ec_words(int n_ec) { return (n_ec + 31) / 32; }
GQB_HD inline int ec_stride(int n_ec) { return (ec_words(n_ec) + 3) & ~3; }

// words from the blob start to the 16-byte aligned rel_ecs rows
GQB_HD inline uint32_t rel_ecs_offset(int n_ec, int n_sels, int n_fks) {
    const uint32_t w = (uint32_t)(sizeof(DevHeader) / 4 + 2 * n_ec + n_sels + n_fks + n_fks * (sizeof(DevVar) / 4));
    return (w + 3u) & ~3u;
}

GQB_HD inline DevInfoView make_view(const void *blob) {
    DevInfoView v;
    v.h = reinterpret_cast<const DevHeader *>(blob);
    const uint32_t *p = reinterpret_cast<const uint32_t *>(v.h + 1);
    v.ec_relids = p;
    p += v.h->n_ec;
    v.ec_off = p;
    p += v.h->n_ec;
    v.sels = reinterpret_cast<const float *>(p);
    p += v.h->n_sels;
    v.fks = p;
    p += v.h->n_fks;
    v.vars = reinterpret_cast<const DevVar *>(p);
    v.rel_ecs = reinterpret_cast<const uint32_t *>(v.h) + rel_ecs_offset(v.h->n_ec, v.h->n_sels, v.h->n_fks);
    v.pair_sel = reinterpret_cast<const float *>(v.rel_ecs + v.h->n * ec_stride(v.h->n_ec));
    v.plain = reinterpret_cast<const uint32_t *>(v.pair_sel + ((2 * v.h->n_ec + 3) & ~3));
    return v;
}

GQB_HD inline uint32_t blob_words_for(int n, int n_ec, int n_sels, int n_fks) {
    return rel_ecs_offset(n_ec, n_sels, n_fks) + (uint32_t)(n * ec_stride(n_ec) + ((2 * n_ec + 3) & ~3) +
                                                            ec_stride(n_ec));
}

// fills DevInfoView::rel_ecs from the class member masks (compact bits)
GQB_HD inline void fill_rel_ecs(const DevInfoView &v, int n) {
    uint32_t *out = const_cast<uint32_t *>(v.rel_ecs);
    const int ecs = ec_stride(v.h->n_ec);
    for (int i = 0; i < n * ecs; i++) out[i] = 0u;
    for (int e = 0; e < v.h->n_ec; e++)
        for (uint32_t m = v.ec_relids[e]; m; m &= m - 1u) {
            int r = 0;
            while (!((m >> r) & 1u)) r++;
            out[r * ecs + e / 32] |= 1u << (e % 32);
        }
}

// fills DevInfoView::pair_sel, DevInfoView::plain and DevHeader::all_pairs
// from the class arrays
// and DevHeader::fksel (after those are written): ec_selectivity
// (gpuqo_row_estimation.cuh:49-88) of a two-member class {x < y} is the FK
// selectivity of the outer member's key into the inner one, else of the
// inner member's key into the outer one, else the class's stored
// selectivity; it selects a value and does no arithmetic, so the table holds
// exactly what the per-pair evaluation would compute.
GQB_HD inline void fill_pair_sel(const DevInfoView &v) {
    DevHeader *h = const_cast<DevHeader *>(v.h);
    float *ps = const_cast<float *>(v.pair_sel);
    for (int w = 0; w < ec_stride(h->n_ec); w++) const_cast<uint32_t *>(v.plain)[w] = 0u;
    uint32_t all = 1u;
    for (int i = 0; i < h->n_ec; i++) {
        const uint32_t rr = v.ec_relids[i];
        uint32_t m = rr;
        int cnt = 0, x = -1, y = -1;
        for (int r = 0; m; r++, m >>= 1)
            if (m & 1u) {
                if (cnt == 0) x = r;
                y = r;
                cnt++;
            }
        if (cnt != 2) {
            all = 0u;
            ps[2 * i] = ps[2 * i + 1] = __builtin_nanf("");
            continue;
        }
        const int off_f = (int)(v.ec_off[i] & 0xFFFFu), off_s = (int)(v.ec_off[i] >> 16);
        const bool fk_xy = (v.fks[off_f + 0] >> y) & 1u;   // member x's key matches y
        const bool fk_yx = (v.fks[off_f + 1] >> x) & 1u;   // member y's key matches x
        const float sel = v.sels[off_s];
        ps[2 * i] = fk_xy ? h->fksel[y] : (fk_yx ? h->fksel[x] : sel);
        ps[2 * i + 1] = fk_yx ? h->fksel[x] : (fk_xy ? h->fksel[y] : sel);
        bool plain = true;
        for (int j = 0; j < 2; j++) {
            const DevVar &dv = v.vars[off_f + j];
            plain = plain && (dv.flags & (1u | kVarMcvRatio)) == 0u && (dv.flags & kVarNoDistinct) != 0u &&
                    dv.mcvfreq == 0.0f;
        }
        if (plain) const_cast<uint32_t *>(v.plain)[i / 32] |= 1u << (i % 32);
    }
    h->all_pairs = (h->n_ec > 0) ? all : 0u;
}

}  // namespace gqb
