// dp_device.cuh - device-side data layout and per-pair arithmetic of the
// B200 join-order DP (DPsub / MPDP).
//
// Relation sets on the device use COMPACT masks: bit i = relation i after the
// BFS relabelling (the reference's Postgres-style masks use bit i+1; the shift
// preserves every order the algorithm depends on: lowest bit, pdep order,
// integer order of subsets).
//
// Floating point follows the reference's cost model operation by operation
// (src/backend/optimizer/gpuqo/gpuqo_cost.cuh, gpuqo_cost_postgres.cuh,
// gpuqo_row_estimation.cuh).  This file must be compiled with -fmad=false:
// the reference's CPU engines never fuse a multiply with an add.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dp_layout.h"

namespace gqb {

// ---------------------------------------------------------------------------
// bit helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lowest(uint32_t x) { return x & (0u - x); }
__device__ __forceinline__ int lowest_idx(uint32_t x) { return __ffs(x) - 1; }
__device__ __forceinline__ int popc(uint32_t x) { return __popc(x); }

// gpuqo_bitmapset.cuh:302-305: next subset of `set` after `sub` (pdep order)
__device__ __forceinline__ uint32_t next_subset(uint32_t sub, uint32_t set) { return set & (sub - set); }

// deposit the low bits of `val` into the set bits of `mask`
__device__ __forceinline__ uint32_t pdep32(uint32_t val, uint32_t mask) {
    uint32_t r = 0;
    while (mask && val) {
        uint32_t low = mask & (0u - mask);
        if (val & 1u) r |= low;
        val >>= 1;
        mask ^= low;
    }
    return r;
}

// gpuqo_filter.cuh:119-147: closure of `from` inside `subset`
__device__ __forceinline__ uint32_t grow(uint32_t from, uint32_t subset, const uint32_t *adj) {
    uint32_t V = 0, N = from;
    while (N) {
        int i = __ffs(N) - 1;
        V |= 1u << i;
        N = (N | adj[i]) & subset & ~V;
    }
    return V;
}

// gpuqo_filter.cuh:149-160
__device__ __forceinline__ bool is_connected(uint32_t s, const uint32_t *adj) {
    if (!s) return false;
    return grow(lowest(s), s, adj) == s;
}

// float -> int as the reference's x86-64 host build converts it
// (cvttss2si: truncation, INT_MIN when out of range or NaN).  The device's
// own conversion saturates instead, so it is emulated.
__device__ __forceinline__ int f2i_x86(float f) {
    if (!(f > -2147483649.0f && f < 2147483648.0f)) return (int)0x80000000;
    return __float2int_rz(f);
}

__device__ __forceinline__ int ceil_log2_l(long long num) {
    int res = 63 - __clzll(num);
    if ((1LL << res) == num) return res;
    return res + 1;
}

// order-preserving map of a float to uint32 (NaN handled by the caller);
// -0.0 is folded to +0.0 because the reference compares with '<'
__device__ __forceinline__ uint32_t ord_float(float f) {
    if (f == 0.0f) f = 0.0f;
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// ---------------------------------------------------------------------------
// cost model pieces (gpuqo_cost_postgres.cuh)
// ---------------------------------------------------------------------------
struct RelVal {
    float rows, startup, total;
    int width;
    uint32_t hz;   // packed hash table size of this set as an inner side, 0 if not stored
};

// Memo width word.  With DevHeader::hz_packed the low 21 bits hold the width,
// bit 21 marks a stored hash table size, bits 22-26 log2(numbuckets) and
// bits 27-31 log2(numbatches) of ExecChooseHashTableSize for the set as an
// inner relation (a function of its rows and width only), computed once when
// the entry is written instead of once per pair that reads it.
constexpr uint32_t kWidthBits = 21;
constexpr uint32_t kWidthMask = (1u << kWidthBits) - 1u;

// a memo entry already loaded (see load_rel)
__device__ __forceinline__ RelVal unpack_rel(const float4 v, uint32_t packed) {
    RelVal r;
    r.rows = v.x;
    r.startup = v.y;
    r.total = v.z;
    const uint32_t w = __float_as_uint(v.w);
    r.width = packed ? (int)(w & kWidthMask) : (int)w;
    r.hz = packed ? (w >> kWidthBits) : 0u;
    return r;
}

__device__ __forceinline__ RelVal load_rel(const float4 *memo, uint32_t s, uint32_t packed) {
    return unpack_rel(__ldcg(memo + s), packed);
}

// :850-862
__device__ __forceinline__ float clamp_row_est(float nrows) {
    return nrows <= 1.0f ? 1.0f : rintf(nrows);
}

// :820-841 (MAXALIGN with MAXIMUM_ALIGNOF 8, RELATION_OVERHEAD 24, BLCKSZ 8192)
__device__ __forceinline__ float relation_byte_size(float tuples, int width) {
    unsigned long long a = ((unsigned long long)(long long)width + 7ull) & ~7ull;
    return tuples * (float)(a + 24ull);
}
__device__ __forceinline__ float page_size(float tuples, int width) {
    return ceilf(relation_byte_size(tuples, width) / 8192.0f);
}

struct Htsz {
    int numbuckets, numbatches;
};

// :480-621 ExecChooseHashTableSize
__device__ __forceinline__ Htsz exec_choose_hash_table_size(float ntuples, int tupwidth, int work_mem) {
    Htsz res;
    res.numbatches = 1;
    if (ntuples <= 0.0f) ntuples = 1000.0f;
    int tupsize = 32 + (int)(((unsigned long long)(long long)tupwidth + 7ull) & ~7ull);
    float inner_rel_bytes = ntuples * (float)tupsize;
    long long hash_table_bytes = (long long)work_mem * 1024LL;
    float space_allowed = (float)hash_table_bytes;
    long long skew_table_bytes = hash_table_bytes * 2 / 100;
    // num_skew_mcvs = skew_table_bytes / (tupsize + 84) > 0  <=>  skew >= tupsize + 84
    if (skew_table_bytes >= (long long)(tupsize + 84)) hash_table_bytes -= skew_table_bytes;
    long long max_pointers = (long long)(space_allowed / 8.0f);
    {
        unsigned long long a = (unsigned long long)max_pointers, b = 0x3fffffffULL / 8ULL;
        max_pointers = (long long)(a < b ? a : b);
    }
    long long mppow2 = 1LL << ceil_log2_l(max_pointers);
    if (max_pointers != mppow2) max_pointers = mppow2 / 2;
    if (max_pointers > (long long)(2147483647 / 2)) max_pointers = 2147483647 / 2;
    float dbuckets = ceilf(ntuples / 1.0f);
    dbuckets = fminf(dbuckets, (float)max_pointers);
    res.numbuckets = (int)dbuckets;
    if (res.numbuckets < 1024) res.numbuckets = 1024;
    res.numbuckets = 1 << ceil_log2_l(res.numbuckets);
    long long bucket_bytes = 8LL * res.numbuckets;
    if (inner_rel_bytes + (float)bucket_bytes > (float)hash_table_bytes) {
        long long bucket_size = (long long)tupsize + 8LL;
        long long q = (hash_table_bytes < 0x100000000LL && bucket_size < 0x100000000LL)
                          ? (long long)((uint32_t)hash_table_bytes / (uint32_t)bucket_size)
                          : hash_table_bytes / bucket_size;
        long long lbuckets = 1LL << ceil_log2_l(q);
        if (lbuckets > max_pointers) lbuckets = max_pointers;
        res.numbuckets = (int)lbuckets;
        res.numbuckets = 1 << ceil_log2_l(res.numbuckets);
        bucket_bytes = 8LL * res.numbuckets;
        float dbatch = ceilf(inner_rel_bytes / (float)(hash_table_bytes - bucket_bytes));
        dbatch = fminf(dbatch, (float)max_pointers);
        int minbatch = (int)dbatch;
        int p2 = 1 << ceil_log2_l(minbatch);
        res.numbatches = p2 > 2 ? p2 : 2;
    }
    return res;
}

// classes of a join found through DevInfoView::rel_ecs up to this many words
// of 32 classes (1024 classes); beyond, every class is scanned
constexpr int kMaxEcWords = 32;

// 1 / v for v = +-2^m, exactly (sign and exponent bits); the bucket counts
// of the cost model are products of powers of two, or INT_MIN after the x86
// conversion of 2^31 and above.  Equal to the IEEE quotient, which is exact.
__device__ __forceinline__ float recip_pow2(int v) {
    const uint32_t a = v < 0 ? 0u - (uint32_t)v : (uint32_t)v;
    if (a == 0u || (a & (a - 1u)) != 0u) return 1.0f / (float)v;   // not a power of two
    const uint32_t m = 31u - (uint32_t)__clz(a);
    return __uint_as_float((v < 0 ? 0x80000000u : 0u) | ((127u - m) << 23));
}

// :705-787 __estimate_hash_bucketsize; the relation-only terms come from
// devvar_bucket_terms, only the bucket count depends on the pair
__device__ __forceinline__ float bucketsize_one(const DevVar &v, int nbuckets) {
    if (v.flags & kVarNoDistinct) return 0.1f;
    float estfract = (v.bs_nd > (float)nbuckets) ? recip_pow2(nbuckets) : v.bs_inv_nd;
    if (v.flags & kVarMcvRatio) estfract *= v.bs_mcv_ratio;
    if (estfract < 1.0e-6f) estfract = 1.0e-6f;
    else if (estfract > 1.0f) estfract = 1.0f;
    return estfract;
}

struct Extra {
    bool inner_unique;
    bool indexed_join_quals;
    float joinrows, outer_match_frac, match_count;
};

// :114-279 cost_nestloop; (n_quals, per_tuple) is cost_qual_eval(inner, outer)
__device__ __forceinline__ void cost_nestloop(const DevHeader &h, const RelVal &outer, float inner_rows,
                                              float inner_startup, float inner_total, const Extra &extra,
                                              float qual_per_tuple, float &out_startup, float &out_total) {
    float startup_cost = 0.0f, run_cost = 0.0f;
    float outer_path_rows = outer.rows, inner_path_rows = inner_rows, ntuples;
    if (!h.enable_nestloop) startup_cost += h.disable_cost;
    startup_cost += inner_startup + outer.startup;
    run_cost += outer.total - outer.startup;
    if (outer_path_rows > 1.0f) run_cost += (outer_path_rows - 1.0f) * inner_startup;
    float inner_run_cost = inner_total - inner_startup;
    float inner_rescan_run_cost = inner_run_cost;
    if (extra.inner_unique) {
        float outer_matched_rows = rintf(outer_path_rows * extra.outer_match_frac);
        float outer_unmatched_rows = outer_path_rows - outer_matched_rows;
        float inner_scan_frac = 2.0f / (extra.match_count + 1.0f);
        ntuples = outer_matched_rows * inner_path_rows * inner_scan_frac;
        if (extra.indexed_join_quals) {
            run_cost += inner_run_cost * inner_scan_frac;
            if (outer_matched_rows > 1.0f)
                run_cost += (outer_matched_rows - 1.0f) * inner_rescan_run_cost * inner_scan_frac;
            run_cost += outer_unmatched_rows * inner_rescan_run_cost / inner_path_rows;
        } else {
            ntuples += outer_unmatched_rows * inner_path_rows;
            run_cost += inner_run_cost;
            if (outer_unmatched_rows >= 1.0f) outer_unmatched_rows -= 1.0f;
            else outer_matched_rows -= 1.0f;
            if (outer_matched_rows > 0.0f) run_cost += outer_matched_rows * inner_rescan_run_cost * inner_scan_frac;
            if (outer_unmatched_rows > 0.0f) run_cost += outer_unmatched_rows * inner_rescan_run_cost;
        }
    } else {
        run_cost += inner_run_cost;
        if (outer_path_rows > 1.0f) run_cost += (outer_path_rows - 1.0f) * inner_rescan_run_cost;
        ntuples = outer_path_rows * inner_path_rows;
    }
    startup_cost += 0.0f;  // cost_qual_eval startup is always 0
    float cpu_per_tuple = h.cpu_tuple_cost + qual_per_tuple;
    run_cost += cpu_per_tuple * ntuples;
    out_startup = startup_cost;
    out_total = startup_cost + run_cost;
}

// :291-468 cost_hashjoin
__device__ __forceinline__ void cost_hashjoin(const DevHeader &h, const RelVal &outer, const RelVal &inner,
                                              const Extra &extra, int n_quals, float qual_per_tuple,
                                              const Htsz &hz, float bs_bucketsize, float bs_mcvfreq,
                                              float &out_startup, float &out_total) {
    float startup_cost = 0.0f, run_cost = 0.0f, hashjointuples;
    float outer_path_rows = outer.rows, inner_path_rows = inner.rows;
    if (!h.enable_hashjoin) startup_cost += h.disable_cost;
    startup_cost += outer.startup;
    run_cost += outer.total - outer.startup;
    startup_cost += inner.total;
    startup_cost += (h.cpu_operator_cost * (float)n_quals + h.cpu_tuple_cost) * inner_path_rows;
    run_cost += h.cpu_operator_cost * (float)n_quals * outer_path_rows;
    if (hz.numbatches > 1) {
        float outerpages = page_size(outer_path_rows, outer.width);
        float innerpages = page_size(inner_path_rows, inner.width);
        startup_cost += h.seq_page_cost * innerpages;
        run_cost += h.seq_page_cost * (innerpages + 2.0f * outerpages);
    }
    if (relation_byte_size(clamp_row_est(inner_path_rows * bs_mcvfreq), inner.width) >
        (float)((long long)h.work_mem * 1024LL))
        startup_cost += h.disable_cost;
    if (extra.inner_unique) {
        float outer_matched_rows = rintf(outer_path_rows * extra.outer_match_frac);
        float inner_scan_frac = 2.0f / (extra.match_count + 1.0f);
        startup_cost += 0.0f;
        run_cost += qual_per_tuple * outer_matched_rows *
                    clamp_row_est(inner_path_rows * bs_bucketsize * inner_scan_frac) * 0.5f;
        run_cost += qual_per_tuple * (outer_path_rows - outer_matched_rows) *
                    // virtualbuckets = 2^(log2 numbuckets + log2 numbatches): dividing by it is
                    // multiplying by its exact reciprocal (same real value, same rounding)
                    clamp_row_est(inner_path_rows * __uint_as_float(
                                      (127u - (31u - (uint32_t)__clz(hz.numbuckets)) -
                                       (31u - (uint32_t)__clz(hz.numbatches))) << 23)) * 0.05f;
        hashjointuples = outer_matched_rows;
    } else {
        startup_cost += 0.0f;
        run_cost += qual_per_tuple * outer_path_rows * clamp_row_est(inner_path_rows * bs_bucketsize) * 0.5f;
        hashjointuples = extra.joinrows;
    }
    run_cost += h.cpu_tuple_cost * hashjointuples;
    out_startup = startup_cost;
    out_total = startup_cost + run_cost;
}

// gpuqo_row_estimation.cuh:26-45 fkselc_of_ec; returns NaN when no FK applies
__device__ __forceinline__ float fkselc_of_ec(const DevInfoView &d, int off_fk, uint32_t ec, uint32_t outer_rels,
                                              uint32_t inner_rels) {
    uint32_t tmp = outer_rels;
    while (tmp) {
        uint32_t out_id = lowest(tmp);
        int out_idx = popc((out_id - 1u) & ec);
        uint32_t match = inner_rels & d.fks[off_fk + out_idx];
        if (match) {
            return d.h->fksel[lowest_idx(match)];
        }
        tmp &= ~out_id;
    }
    return __int_as_float(0x7fffffff);
}

// gpuqo_row_estimation.cuh:49-88 (for a class that matches both sides)
__device__ __forceinline__ float ec_selectivity(const DevInfoView &d, int i, uint32_t ec, uint32_t ml, uint32_t mr) {
    uint32_t off = d.ec_off[i];
    int off_sels = (int)(off >> 16), off_fks = (int)(off & 0xFFFFu);
    float fk = fkselc_of_ec(d, off_fks, ec, ml, mr);
    if (!isnan(fk)) return fk;
    fk = fkselc_of_ec(d, off_fks, ec, mr, ml);
    if (!isnan(fk)) return fk;
    int size = popc(ec);
    int il = popc((lowest(ml) - 1u) & ec);
    int ir = popc((lowest(mr) - 1u) & ec);
    if (il > ir) { int t = il; il = ir; ir = t; }
    int idx = il * size - il * (il + 1) / 2 + (ir - il - 1);
    return d.sels[off_sels + idx];
}

// width word of a memo entry for a set of this rows and width (see kWidthBits)
__device__ __forceinline__ uint32_t memo_width_word(const DevHeader &h, float rows, int width) {
    if (!h.hz_packed) return (uint32_t)width;
    const Htsz z = exec_choose_hash_table_size(rows, width, h.work_mem);
    const uint32_t lb = 31u - (uint32_t)__clz(z.numbuckets), lt = 31u - (uint32_t)__clz(z.numbatches);
    return (uint32_t)width | (1u << kWidthBits) | (lb << (kWidthBits + 1)) | (lt << (kWidthBits + 6));
}

// memo entry of base relation i (gpuqo_cpu_sequential.cu:80-92)
__device__ __forceinline__ float4 base_entry(const DevHeader &h, int i) {
    return make_float4(h.rows[i], h.startup[i], h.total[i], __uint_as_float(memo_width_word(h, h.rows[i], h.width[i])));
}

// Plain DPsub's enumeration index of the split (L, S - L): cpu_dpsub visits
// the nonempty proper subsets L of S in nextSubset order
// (gpuqo_cpu_dpsub.cu:32-78), i.e. L = pdep(p + 1, S), so p = pext(L, S) - 1.
// Computed over the smaller side (pext(R, S) is the complement within the
// |S| low bits).
__device__ __forceinline__ uint32_t dpsub_index(uint32_t L, uint32_t S) {
    const uint32_t R = S ^ L;
    const bool left = __popc(L) <= __popc(R);
    uint32_t x = left ? L : R, r = 0u;
    while (x) {
        const uint32_t b = x & (0u - x);
        r |= 1u << __popc(S & (b - 1u));
        x ^= b;
    }
    if (!left) {
        const int k = __popc(S);
        r ^= (k == 32) ? 0xFFFFFFFFu : ((1u << k) - 1u);
    }
    return r - 1u;
}

// The block enumeration (MPDP) produces exactly the valid csg-cmp pairs of S:
// all edges between the two connected sides of a valid split lie on common
// cycles, hence in one biconnected block B, and growing the two parts of B
// inside S returns the two sides.  Keying each pair by its plain-DPsub index
// therefore gives cpu_dpsub's first strict minimum (and its first NaN) while
// skipping the invalid subsets DPsub would test.
__device__ __forceinline__ uint32_t key_index(const DevHeader &h, uint32_t c, uint32_t L, uint32_t S) {
    return h.index_order ? dpsub_index(L, S) : c;
}

// ---------------------------------------------------------------------------
// One join evaluation: estimate_join_rows + calc_join_cost + width
// (gpuqo_cpu_common.cuh:169-186 make_join_relation; gpuqo_cost.cuh:81-157).
// All per-equivalence-class passes of the reference (selectivity product,
// cost_qual_eval, is_inner_unique, estimate_hash_bucket_stats) are fused into
// one pass; each quantity is accumulated in the reference's class order, so
// every float result is the reference's.
// ---------------------------------------------------------------------------
template <bool MASKED>
__device__ __forceinline__ RelVal join_eval_t(const DevInfoView &d, uint32_t L, const RelVal &l, uint32_t R,
                                              const RelVal &r, uint32_t ec_mask) {
    const DevHeader &h = *d.h;
    const bool inner_single = (R & (R - 1u)) == 0u;
    // the hash table size depends on the inner side only (stored with its memo
    // entry when hz_packed); needed by the bucket-size estimate in the class loop
    Htsz hz;
    if (r.hz) {
        hz.numbuckets = 1 << ((r.hz >> 1) & 31u);
        hz.numbatches = 1 << (r.hz >> 6);
    } else {
        hz = exec_choose_hash_table_size(r.rows, r.width, h.work_mem);
    }
    int nbuckets = f2i_x86((float)hz.numbuckets * (float)hz.numbatches);

    float sel = 1.0f;
    int n_quals = 0;
    float per_tuple = 0.0f;
    bool inner_unique = false, any_index = false;
    float bucketsize = 1.0f, mcvfreq = 1.0f;
    const int n_ec = h.n_ec;
    // Only classes with a member on each side can match, visited in
    // increasing class order (the reference's order): MASKED, the classes in
    // ec_mask (the split edge of a tree-shaped query); otherwise the classes
    // of L's relations and of R's relations intersected word by word
    // (rel_ecs), or every class when there are more than kMaxEcWords words.
    const int ecw = MASKED ? 1 : ec_words(n_ec);
    const int ecs = ec_stride(n_ec);
    const bool by_mask = MASKED || ecw <= kMaxEcWords;
    uint32_t match[kMaxEcWords];
    if (MASKED) {
        match[0] = ec_mask;
    } else if (by_mask) {
        for (int w = 0; w < ecw; w++) {
            uint32_t cl = 0u, cr = 0u;
            for (uint32_t x = L; x; x &= x - 1u) cl |= d.rel_ecs[lowest_idx(x) * ecs + w];
            for (uint32_t x = R; x; x &= x - 1u) cr |= d.rel_ecs[lowest_idx(x) * ecs + w];
            match[w] = cl & cr;
        }
    }
    int w = 0;
    uint32_t mrem = by_mask ? match[0] : 0u;
    for (int i = 0;; i++) {
        if (by_mask) {
            while (mrem == 0u && ++w < ecw) mrem = match[w];
            if (mrem == 0u) break;
            i = (w << 5) + __ffs(mrem) - 1;
            mrem &= mrem - 1u;
        } else if (i >= n_ec) {
            break;
        }
        uint32_t ec = d.ec_relids[i];
        uint32_t ml = ec & L, mr = ec & R;
        if (!ml || !mr) continue;
        // MASKED: a two-member class with one member on each side; its
        // ec_selectivity for this orientation is tabulated in the header.  A
        // plain class (DevInfoView::plain) takes its pair selectivity, and its
        // inner member's variable would give bucket size 0.1 and MCV
        // frequency 0 without an index: set directly, the member not read.
        const bool plain = (d.plain[i >> 5] >> (i & 31)) & 1u;
        if (MASKED) {
            sel *= h.edge_sel[ml > mr ? 1 : 0][i];
        } else if (plain) {
            const float2 ps = *reinterpret_cast<const float2 *>(d.pair_sel + 2 * i);
            sel *= (lowest(ec) & L) ? ps.x : ps.y;
        } else {
            sel *= ec_selectivity(d, i, ec, ml, mr);
        }
        per_tuple += h.cpu_operator_cost;
        n_quals++;
        if (plain) {
            if (bucketsize > 0.1f) bucketsize = 0.1f;
            if (mcvfreq > 0.0f) mcvfreq = 0.0f;
            continue;
        }
        int off_fks = (int)(d.ec_off[i] & 0xFFFFu);
        uint32_t m = mr;
        bool first = true;
        while (m) {
            uint32_t in_id = lowest(m);
            int in_idx = popc((in_id - 1u) & ec);
            const DevVar v = d.vars[off_fks + in_idx];
            if (first && inner_single) {
                if ((v.flags & 1u) && (v.flags & 2u)) inner_unique = true;
                if (v.flags & 1u) any_index = true;
            }
            first = false;
            float this_bs = bucketsize_one(v, nbuckets);
            if (bucketsize > this_bs) bucketsize = this_bs;
            if (mcvfreq > v.mcvfreq) mcvfreq = v.mcvfreq;
            m &= ~in_id;
        }
    }

    RelVal out;
    float rows = sel * l.rows * r.rows;
    out.rows = rows > 1.0f ? roundf(rows) : 1.0f;
    out.width = l.width + r.width;

    Extra extra;
    extra.inner_unique = inner_unique;
    extra.indexed_join_quals = false;
    extra.joinrows = out.rows;
    // read by the cost functions only for a unique inner side
    extra.outer_match_frac = inner_unique ? out.rows / (l.rows * r.rows) : 0.0f;
    extra.match_count = r.rows;

    float min_s, min_t, s, t;
    cost_nestloop(h, l, r.rows, r.startup, r.total, extra, per_tuple, min_s, min_t);
    if (h.enable_hashjoin) {
        cost_hashjoin(h, l, r, extra, n_quals, per_tuple, hz, bucketsize, mcvfreq, s, t);
        if (t < min_t) { min_s = s; min_t = t; }
    }
    if (any_index && !((h.composite_mask >> lowest_idx(R)) & 1u)) {
        extra.indexed_join_quals = true;
        int w2 = 0;
        uint32_t mrem2 = by_mask ? match[0] : 0u;
        for (int i = 0;; i++) {
            if (by_mask) {
                while (mrem2 == 0u && ++w2 < ecw) mrem2 = match[w2];
                if (mrem2 == 0u) break;
                i = (w2 << 5) + __ffs(mrem2) - 1;
                mrem2 &= mrem2 - 1u;
            } else if (i >= n_ec) {
                break;
            }
            uint32_t ec = d.ec_relids[i];
            uint32_t ml = ec & L, mr = ec & R;
            if (!ml || !mr) continue;
            int off_fks = (int)(d.ec_off[i] & 0xFFFFu);
            int in_idx = popc((lowest(mr) - 1u) & ec);
            const DevVar v = d.vars[off_fks + in_idx];
            if (!(v.flags & 1u)) continue;
            cost_nestloop(h, l, v.idx_rows, v.idx_startup, v.idx_total, extra, per_tuple, s, t);
            if (t < min_t) { min_s = s; min_t = t; }
        }
    }
    out.startup = min_s;
    out.total = min_t;
    return out;
}

__device__ __forceinline__ RelVal join_eval(const DevInfoView &d, uint32_t L, const RelVal &l, uint32_t R,
                                            const RelVal &r) {
    return join_eval_t<false>(d, L, l, R, r, 0u);
}

// ---------------------------------------------------------------------------
// Both orientations of one split in one pass.  Plain DPsub costs every split
// (L, R) and its mirror (R, L); the classes with a member on each side are the
// same for both, so they are found once (rel_ecs rows, 16-byte vector loads)
// and visited once, while every quantity of each orientation is accumulated
// with join_eval_t's operations in join_eval_t's class order, so each result
// equals join_eval's bit for bit.  A two-member class takes its selectivity
// for either orientation from DevInfoView::pair_sel (the value ec_selectivity
// selects, precomputed on the host).
// NW: 16-byte words per rel_ecs row (1: up to 128 classes, 2: up to 256).
// ---------------------------------------------------------------------------
struct SideTerms {
    Htsz hz;
    int nbuckets;
    float sel, bucketsize, mcvfreq;
    bool inner_unique, any_index;
};

__device__ __forceinline__ void side_init(const DevHeader &h, const RelVal &inner, SideTerms &t) {
    if (inner.hz) {
        t.hz.numbuckets = 1 << ((inner.hz >> 1) & 31u);
        t.hz.numbatches = 1 << (inner.hz >> 6);
    } else {
        t.hz = exec_choose_hash_table_size(inner.rows, inner.width, h.work_mem);
    }
    t.nbuckets = f2i_x86((float)t.hz.numbuckets * (float)t.hz.numbatches);
    t.sel = 1.0f;
    t.bucketsize = 1.0f;
    t.mcvfreq = 1.0f;
    t.inner_unique = false;
    t.any_index = false;
}

// one inner member's variable (first: the class's lowest inner member)
__device__ __forceinline__ void side_var(SideTerms &t, const DevVar &v, bool first, bool inner_single) {
    if (first && inner_single) {
        if ((v.flags & 1u) && (v.flags & 2u)) t.inner_unique = true;
        if (v.flags & 1u) t.any_index = true;
    }
    const float this_bs = bucketsize_one(v, t.nbuckets);
    if (t.bucketsize > this_bs) t.bucketsize = this_bs;
    if (t.mcvfreq > v.mcvfreq) t.mcvfreq = v.mcvfreq;
}

// general class of any size: the inner members of one orientation
__device__ __forceinline__ void side_members(const DevInfoView &d, int off_fks, uint32_t ec, uint32_t mi,
                                             bool inner_single, SideTerms &t) {
    bool first = true;
    for (uint32_t m = mi; m; m &= m - 1u) {
        const uint32_t in_id = lowest(m);
        side_var(t, d.vars[off_fks + popc((in_id - 1u) & ec)], first, inner_single);
        first = false;
    }
}

// rows, the cost functions and the index nested loops of one orientation
// (outer O, inner I): the tail of join_eval_t
template <int NW>
__device__ __forceinline__ RelVal side_finish(const DevInfoView &d, uint32_t O, const RelVal &o, uint32_t I,
                                              const RelVal &in, const SideTerms &t, int n_quals, float per_tuple,
                                              const uint32_t (&match)[4 * NW]) {
    const DevHeader &h = *d.h;
    RelVal out;
    const float rows = t.sel * o.rows * in.rows;
    out.rows = rows > 1.0f ? roundf(rows) : 1.0f;
    out.width = o.width + in.width;
    Extra extra;
    extra.inner_unique = t.inner_unique;
    extra.indexed_join_quals = false;
    extra.joinrows = out.rows;
    extra.outer_match_frac = t.inner_unique ? out.rows / (o.rows * in.rows) : 0.0f;
    extra.match_count = in.rows;
    float min_s, min_t, s, c;
    cost_nestloop(h, o, in.rows, in.startup, in.total, extra, per_tuple, min_s, min_t);
    if (h.enable_hashjoin) {
        cost_hashjoin(h, o, in, extra, n_quals, per_tuple, t.hz, t.bucketsize, t.mcvfreq, s, c);
        if (c < min_t) { min_s = s; min_t = c; }
    }
    if (t.any_index && !((h.composite_mask >> lowest_idx(I)) & 1u)) {
        extra.indexed_join_quals = true;
#pragma unroll
        for (int w = 0; w < 4 * NW; w++) {
            for (uint32_t mm = match[w]; mm; mm &= mm - 1u) {
                const int i = (w << 5) + __ffs(mm) - 1;
                const uint32_t ec = d.ec_relids[i];
                const int off_fks = (int)(d.ec_off[i] & 0xFFFFu);
                const DevVar v = d.vars[off_fks + popc((lowest(ec & I) - 1u) & ec)];
                if (!(v.flags & 1u)) continue;
                cost_nestloop(h, o, v.idx_rows, v.idx_startup, v.idx_total, extra, per_tuple, s, c);
                if (c < min_t) { min_s = s; min_t = c; }
            }
        }
    }
    out.startup = min_s;
    out.total = min_t;
    return out;
}

// MASKED (tree-shaped query graph, DevHeader::ec_masked): every class is a
// two-member class on an edge, and the classes of the split edge are ec_mask
template <int NW, bool MASKED>
__device__ __forceinline__ void join_eval_mirror_w(const DevInfoView &d, uint32_t L, const RelVal &l, uint32_t R,
                                                   const RelVal &r, uint32_t ec_mask, RelVal &out_lr,
                                                   RelVal &out_rl) {
    const DevHeader &h = *d.h;
    // classes with a member in L and one in R, 32 per word, in class order
    uint32_t match[4 * NW];
    if (MASKED) {
        match[0] = ec_mask;
#pragma unroll
        for (int w = 1; w < 4 * NW; w++) match[w] = 0u;
    } else {
        uint32_t cl[4 * NW], cr[4 * NW];
#pragma unroll
        for (int w = 0; w < 4 * NW; w++) cl[w] = cr[w] = 0u;
        for (uint32_t x = L; x; x &= x - 1u) {
            const uint4 *row = reinterpret_cast<const uint4 *>(d.rel_ecs + lowest_idx(x) * (4 * NW));
#pragma unroll
            for (int j = 0; j < NW; j++) {
                const uint4 a = row[j];
                cl[4 * j] |= a.x;
                cl[4 * j + 1] |= a.y;
                cl[4 * j + 2] |= a.z;
                cl[4 * j + 3] |= a.w;
            }
        }
        for (uint32_t x = R; x; x &= x - 1u) {
            const uint4 *row = reinterpret_cast<const uint4 *>(d.rel_ecs + lowest_idx(x) * (4 * NW));
#pragma unroll
            for (int j = 0; j < NW; j++) {
                const uint4 a = row[j];
                cr[4 * j] |= a.x;
                cr[4 * j + 1] |= a.y;
                cr[4 * j + 2] |= a.z;
                cr[4 * j + 3] |= a.w;
            }
        }
#pragma unroll
        for (int w = 0; w < 4 * NW; w++) match[w] = cl[w] & cr[w];
    }
    SideTerms lr, rl;   // (outer L, inner R) and (outer R, inner L)
    side_init(h, r, lr);
    side_init(h, l, rl);
    const bool r_single = (R & (R - 1u)) == 0u, l_single = (L & (L - 1u)) == 0u;
    int n_quals = 0;
    float per_tuple = 0.0f;
    // the words are visited in order through a shifting window, so that the
    // match words stay in registers
    uint32_t win[4 * NW];
#pragma unroll
    for (int w = 0; w < 4 * NW; w++) win[w] = match[w];
    // every matching class plain (DevInfoView::plain): only the selectivities
    // and the qual count depend on the classes; the bucket size is 0.1 and
    // the MCV frequency 0 once any class matched, exactly what the general
    // loop below computes for such classes
    bool all_plain = !MASKED || (ec_mask & ~d.plain[0]) == 0u;   // MASKED: at most 32 classes
    if (!MASKED) {
        const uint4 *pl = reinterpret_cast<const uint4 *>(d.plain);
#pragma unroll
        for (int j = 0; j < NW; j++) {
            const uint4 p4 = pl[j];
            all_plain = all_plain && (match[4 * j] & ~p4.x) == 0u && (match[4 * j + 1] & ~p4.y) == 0u &&
                        (match[4 * j + 2] & ~p4.z) == 0u && (match[4 * j + 3] & ~p4.w) == 0u;
        }
    }
    if (all_plain) {
#pragma unroll 1
        for (int base = 0; base < (MASKED ? 32 : 128 * NW); base += 32) {
            for (uint32_t mm = win[0]; mm; mm &= mm - 1u) {
                const int i = base + __ffs(mm) - 1;
                const bool lo_left = (lowest(d.ec_relids[i]) & L) != 0u;
                const float2 ps = *reinterpret_cast<const float2 *>(d.pair_sel + 2 * i);
                lr.sel *= lo_left ? ps.x : ps.y;
                rl.sel *= lo_left ? ps.y : ps.x;
                per_tuple += h.cpu_operator_cost;
                n_quals++;
            }
#pragma unroll
            for (int w = 0; w + 1 < 4 * NW; w++) win[w] = win[w + 1];
            win[4 * NW - 1] = 0u;
        }
        if (n_quals > 0) {
            lr.bucketsize = rl.bucketsize = 0.1f;
            lr.mcvfreq = rl.mcvfreq = 0.0f;
        }
        out_lr = side_finish<NW>(d, L, l, R, r, lr, n_quals, per_tuple, match);
        out_rl = side_finish<NW>(d, R, r, L, l, rl, n_quals, per_tuple, match);
        return;
    }
#pragma unroll 1
    for (int base = 0; base < (MASKED ? 32 : 128 * NW); base += 32) {
        for (uint32_t mm = win[0]; mm; mm &= mm - 1u) {
            const int i = base + __ffs(mm) - 1;
            const uint32_t ec = d.ec_relids[i];
            const int off_fks = (int)(d.ec_off[i] & 0xFFFFu);
            if (MASKED || popc(ec) == 2) {
                // one member on each side; lo_left: the lower member is in L
                const bool lo_left = (lowest(ec) & L) != 0u;
                const float2 ps = *reinterpret_cast<const float2 *>(d.pair_sel + 2 * i);
                lr.sel *= lo_left ? ps.x : ps.y;
                rl.sel *= lo_left ? ps.y : ps.x;
                per_tuple += h.cpu_operator_cost;
                n_quals++;
                side_var(lr, d.vars[off_fks + (lo_left ? 1 : 0)], true, r_single);
                side_var(rl, d.vars[off_fks + (lo_left ? 0 : 1)], true, l_single);
            } else {
                const uint32_t ml = ec & L, mr = ec & R;
                lr.sel *= ec_selectivity(d, i, ec, ml, mr);
                rl.sel *= ec_selectivity(d, i, ec, mr, ml);
                per_tuple += h.cpu_operator_cost;
                n_quals++;
                side_members(d, off_fks, ec, mr, r_single, lr);
                side_members(d, off_fks, ec, ml, l_single, rl);
            }
        }
#pragma unroll
        for (int w = 0; w + 1 < 4 * NW; w++) win[w] = win[w + 1];
        win[4 * NW - 1] = 0u;
    }
    out_lr = side_finish<NW>(d, L, l, R, r, lr, n_quals, per_tuple, match);
    out_rl = side_finish<NW>(d, R, r, L, l, rl, n_quals, per_tuple, match);
}

// (L, R) and (R, L) of a split edge of a tree-shaped query graph (the tree
// kernels' edge decode): MASKED reads only the edge's classes (ec_mask)
template <bool MASKED>
__device__ __forceinline__ void join_eval_mirror_tree(const DevInfoView &d, uint32_t L, const RelVal &l, uint32_t R,
                                                      const RelVal &r, uint32_t ec_mask, RelVal &out_lr,
                                                      RelVal &out_rl) {
    if (MASKED) {
        join_eval_mirror_w<1, true>(d, L, l, R, r, ec_mask, out_lr, out_rl);
    } else {
        // classes off the tree's edges: one orientation after the other (the
        // fused general pass needs more registers than the tree kernels have)
        out_lr = join_eval(d, L, l, R, r);
        out_rl = join_eval(d, R, r, L, l);
    }
}

// (L, R) and (R, L); classes beyond 256 take two join_eval calls
__device__ __forceinline__ void join_eval_mirror(const DevInfoView &d, uint32_t L, const RelVal &l, uint32_t R,
                                                 const RelVal &r, RelVal &out_lr, RelVal &out_rl) {
    const int n_ec = d.h->n_ec;
    if (n_ec <= 128) {
        join_eval_mirror_w<1, false>(d, L, l, R, r, 0u, out_lr, out_rl);
    } else if (n_ec <= 256) {
        join_eval_mirror_w<2, false>(d, L, l, R, r, 0u, out_lr, out_rl);
    } else {
        out_lr = join_eval(d, L, l, R, r);
        out_rl = join_eval(d, R, r, L, l);
    }
}

// ---------------------------------------------------------------------------
// Biconnected blocks of a connected set, in the output order of the
// reference's iterative Hopcroft-Tarjan (gpuqo_cpu_dpsub_bicc.cu:65-170):
// DFS from the lowest relation, neighbours in increasing index order, a block
// emitted when returning from child v to u with low[v] >= disc[u].  A vertex
// stack replaces the reference's edge stack; both yield the same vertex sets
// in the same order.  prefix[b] = number of candidate pairs in blocks < b
// (each block b contributes 2^|b| - 2); sub[b] = vertices of the DFS subtree
// of the block's child end v.  For a 2-vertex block {u, v} (a bridge) the two
// sides of the split are exactly sub[b] and S - sub[b], which is what the
// reference's grow() calls return for it (gpuqo_cpu_dpsub_bicc.cu:188-195).
// ---------------------------------------------------------------------------
// Two index spaces per set: the reference's (prefix/total: block b owns the
// 2^|b| - 2 indices of its subsets, in nextSubset order; candidates are keyed
// and tie-broken by it) and the enumerated one (eprefix/etotal): a block that
// is a simple cycle of four or more relations enumerates only its
// |b|(|b| - 1) arcs, the only subsets with both sides connected.
struct Blocks {
    int nb;
    uint32_t total;               // sum of 2^|b| - 2
    uint32_t etotal;              // candidates enumerated
    uint32_t cyc;                 // bit b: block b is a simple cycle of 4+ relations
    uint32_t mask[kMaxRels];
    uint32_t sub[kMaxRels];
    uint32_t prefix[kMaxRels + 1];
    uint32_t eprefix[kMaxRels + 1];
};

// pext: the bits of x at the positions of mask, packed (x within mask)
__device__ __forceinline__ uint32_t pext32(uint32_t x, uint32_t mask) {
    uint32_t r = 0u;
    for (; x; x &= x - 1u) r |= 1u << __popc(mask & ((x & (0u - x)) - 1u));
    return r;
}

__device__ __forceinline__ void find_blocks(uint32_t S, const uint32_t *adj, Blocks &B) {
    uint8_t disc[kMaxRels], low[kMaxRels], parent[kMaxRels];
    uint8_t stk_u[kMaxRels];
    uint32_t stk_e[kMaxRels];
    uint32_t desc[kMaxRels];
    uint8_t vstk[kMaxRels];
    int sp = 0, vsp = 0, t = 0;
    uint32_t visited = 0;
    B.nb = 0;
    B.total = 0;
    B.etotal = 0;
    B.cyc = 0;
    int root = lowest_idx(S);
    visited |= 1u << root;
    disc[root] = (uint8_t)t++;
    low[root] = 255;
    parent[root] = 255;
    desc[root] = 1u << root;
    vstk[vsp++] = (uint8_t)root;
    stk_u[sp] = (uint8_t)root;
    stk_e[sp] = adj[root] & S;
    sp++;
    while (sp > 0) {
        int u = stk_u[sp - 1];
        uint32_t e = stk_e[sp - 1];
        if (e == 0) {
            sp--;
            if (sp > 0) {
                int p = stk_u[sp - 1];
                if (low[u] >= disc[p]) {
                    uint32_t blk = 1u << p;
                    int w;
                    do {
                        w = vstk[--vsp];
                        blk |= 1u << w;
                    } while (w != u);
                    const uint32_t m = (uint32_t)popc(blk);
                    bool cycle = m >= 4u;
                    for (uint32_t x = blk; cycle && x; x &= x - 1u) cycle = popc(adj[lowest_idx(x)] & blk) == 2;
                    B.prefix[B.nb] = B.total;
                    B.eprefix[B.nb] = B.etotal;
                    if (cycle) B.cyc |= 1u << B.nb;
                    B.sub[B.nb] = desc[u];
                    B.mask[B.nb++] = blk;
                    B.total += (1u << m) - 2u;
                    B.etotal += cycle ? m * (m - 1u) : (1u << m) - 2u;
                }
                if (low[u] < low[p]) low[p] = low[u];
                desc[p] |= desc[u];
                stk_e[sp - 1] &= ~(1u << u);
            }
            continue;
        }
        int v = lowest_idx(e);
        if (!((visited >> v) & 1u)) {
            visited |= 1u << v;
            parent[v] = (uint8_t)u;
            disc[v] = (uint8_t)t++;
            low[v] = 255;
            desc[v] = 1u << v;
            vstk[vsp++] = (uint8_t)v;
            stk_u[sp] = (uint8_t)v;
            stk_e[sp] = adj[v] & S;
            sp++;
        } else {
            if (parent[u] != v && disc[v] < disc[u]) {
                if (disc[v] < low[u]) low[u] = disc[v];
            }
            stk_e[sp - 1] = e & ~(1u << v);
        }
    }
    B.prefix[B.nb] = B.total;
    B.eprefix[B.nb] = B.etotal;
}

// Arcs of one cycle block (m relations) in O(1).  The cycle is walked from
// its lowest relation towards that relation's lower neighbour; pre[i] holds
// the first i relations of the walk (filled once per block).  Arc j starts at
// walk position s = j / (m - 1) and has length j % (m - 1) + 1, wrapping
// around; every nonempty proper connected subset of a cycle is one arc.
struct CycleCache {
    int b = -1;                   // block the prefixes belong to
    uint32_t set = 0u;            // ... of this set
    uint32_t m = 0u;
    uint32_t pre[kMaxRels + 1];
};

__device__ __forceinline__ uint32_t cached_arc(CycleCache &cc, uint32_t S, int b, uint32_t blk, const uint32_t *adj,
                                               uint32_t j) {
    if (cc.b != b || cc.set != S) {
        cc.b = b;
        cc.set = S;
        cc.m = (uint32_t)__popc(blk);
        int v = __ffs(blk) - 1;
        int prev = 31 - __clz(adj[v] & blk);
        cc.pre[0] = 0u;
        for (uint32_t i = 0; i < cc.m; i++) {
            cc.pre[i + 1] = cc.pre[i] | (1u << v);
            const int nx = __ffs(adj[v] & blk & ~(1u << prev)) - 1;
            prev = v;
            v = nx;
        }
    }
    const uint32_t m = cc.m, s = j / (m - 1u), e = s + j % (m - 1u) + 1u;
    return e <= m ? (cc.pre[e] ^ cc.pre[s]) : ((cc.pre[m] ^ cc.pre[s]) | cc.pre[e - m]);
}

// Enumerated candidate c of set S with blocks B (see Blocks): block b and its
// subset lb (for a cycle block an arc, otherwise the (c - eprefix[b] + 1)-th
// subset in nextSubset order); left/right are the reference's grow() results
// and key the candidate's reference index prefix[b] + pext(lb, block) - 1.
// `b` is the caller's cursor (c must not decrease between calls).
__device__ __forceinline__ bool mpdp_candidate(uint32_t S, const Blocks &B, const uint32_t *adj, uint32_t c, int &b,
                                               uint32_t &L, uint32_t &R, uint32_t &key, CycleCache &cc) {
    while (b + 1 < B.nb && B.eprefix[b + 1] <= c) b++;
    const uint32_t blk = B.mask[b];
    const uint32_t j = c - B.eprefix[b];
    if (popc(blk) == 2) {
        // bridge {u, v}: j = 0 -> lb = lowest vertex, j = 1 -> the other
        const uint32_t lo = lowest(blk);
        const uint32_t lb = (j == 0u) ? lo : (blk ^ lo);
        const uint32_t sub = B.sub[b];
        if (lb & sub) {
            L = sub;
            R = S ^ sub;
        } else {
            L = S ^ sub;
            R = sub;
        }
        key = B.prefix[b] + j;
        return true;
    }
    uint32_t lb;
    if ((B.cyc >> b) & 1u) {
        lb = cached_arc(cc, S, b, blk, adj, j);
        key = B.prefix[b] + pext32(lb, blk) - 1u;
        if (blk == S) {   // the set is the cycle: arc and complement are the two sides
            L = lb;
            R = S ^ lb;
            return true;
        }
    } else {
        lb = pdep32(j + 1u, blk);
        key = B.prefix[b] + j;
    }
    const uint32_t rb = blk ^ lb;
    L = grow(lowest(lb), S & ~rb, adj);
    R = grow(lowest(rb), S & ~lb, adj);
    return (L | R) == S;
}

}  // namespace gqb
