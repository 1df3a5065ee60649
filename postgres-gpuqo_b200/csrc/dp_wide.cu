// dp_wide.cu - exact DP of 32 to 63 relations (after the BFS relabelling).
//
// The reference plans up to 63 relations exactly with 64-bit relation sets
// and a hash-table memo (gpuqo_main_internal.cu:177-185, Bitmapset64;
// gpuqo_hashtable.cuh:121-166).  The dense memo of the main engine stops at
// 31 relations (2^n entries); beyond, only the connected sets are stored:
//   * the host enumerates the connected sets level by level (extension by a
//     neighbour, deduplicated) - the graphs planned exactly at this size are
//     sparse, with thousands to millions of connected sets, and the count is
//     checked against the memo's capacity before anything is allocated;
//   * k_wide_insert builds a device open-addressing table (64-bit keys,
//     atomicCAS, linear probing) from each set to its slot; the memo is
//     indexed by slot: (rows, startup, total, width word) and the outer side;
//   * per level, k_wide_eval costs every connected set with one warp: the
//     set's biconnected blocks (the reference's DFS order), every candidate
//     split of every block grown to a csg-cmp pair, both sides looked up in
//     the table, join_eval_w's cost, and a warp reduction of
//     (cost, enumeration index) with 64-bit indices - the MPDP index
//     (gpuqo_cpu_dpsub_bicc.cu:46-236), or for plain DPsub the index of the
//     split in cpu_dpsub's subset order (gpuqo_cpu_dpsub.cu:32-78), which
//     selects the same first strict minimum over the valid pairs only.
// The plan is read back from the memo on the host.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <unordered_set>
#include <vector>

#include "dp_device.cuh"
#include "dp_engine.h"
#include "gpuqo_b200.h"
#include "host_info.h"

extern "C" int gpuqo_b200_device_memory_mb;
extern "C" int gpuqo_b200_sparse_host_list;

namespace gqb {

namespace {

constexpr uint32_t kFullW = 0xFFFFFFFFu;
constexpr int kWideBlock = 256;
constexpr int kWideMaxRels = 63;
constexpr uint64_t kWideMaxCandidates = 1ull << 24;   // candidate splits of one set
constexpr uint64_t kWideMaxTotal = 1ull << 35;        // candidate splits of the whole DP

// planner info on the device (global memory; read through the read-only path)
struct WideInfo {
    DevHeader h;                       // cost parameters (cost_nestloop / cost_hashjoin / memo_width_word)
    int n, n_ec;
    uint64_t composite;                // relations that are composite entries (IDP sub-problems)
    uint64_t adj[64];
    float rows[64], tuples[64], startup[64], total[64], fksel[64];
    int width[64];
    const uint64_t *ec_relids;         // [n_ec]
    const uint32_t *ec_off;            // [n_ec] off_sels << 16 | off_fks
    const float *sels;                 // [n_sels]
    const uint64_t *fks;               // [n_fks]
    const DevVar *vars;                // [n_fks]
    // [n_ec] per class: the selectivity with its lower member outer, with its
    // higher member outer, and whether it is plain (two members whose
    // variables carry no statistics and no index: bucket size 0.1, MCV
    // frequency 0); w unused
    const float4 *pair;
    // a tree whose classes all have two members on an edge (at most 64
    // classes): edge_cls[v] = the classes on the edge between v and its
    // parent in the tree rooted at relation 0
    int edge_masked;
    uint64_t edge_cls[64];
    // at most 64 classes: rel_cls[v] = the classes with a member v; a split
    // (L, R) matches the classes in (OR over L) & (OR over R)
    int rel_masked;
    uint64_t rel_cls[64];
};
constexpr size_t kWideInfoBytes = (sizeof(WideInfo) + 15) & ~size_t(15);

__device__ __forceinline__ uint64_t lowest64(uint64_t x) { return x & (0ull - x); }
__device__ __forceinline__ int lowest_idx64(uint64_t x) { return __ffsll((long long)x) - 1; }

__device__ __forceinline__ uint64_t grow64(uint64_t from, uint64_t subset, const uint64_t *adj) {
    uint64_t V = 0, N = from;
    while (N) {
        const int i = lowest_idx64(N);
        V |= 1ull << i;
        N = (N | adj[i]) & subset & ~V;
    }
    return V;
}

__device__ __forceinline__ uint64_t pdep64(uint64_t val, uint64_t mask) {
    uint64_t r = 0;
    while (mask && val) {
        const uint64_t low = lowest64(mask);
        if (val & 1ull) r |= low;
        val >>= 1;
        mask ^= low;
    }
    return r;
}

__device__ __forceinline__ uint64_t pext64(uint64_t x, uint64_t mask) {
    uint64_t r = 0;
    for (; x; x &= x - 1ull) r |= 1ull << __popcll(mask & (lowest64(x) - 1ull));
    return r;
}

// cpu_dpsub's index of the split (L, S - L): L = pdep(p + 1, S)
__device__ __forceinline__ uint64_t dpsub_index64(uint64_t L, uint64_t S) { return pext64(L, S) - 1ull; }

// biconnected blocks of S in the reference's DFS output order (find_blocks on
// 64-bit sets); prefix: the reference's candidate indices (2^|b| - 2 per
// block), eprefix: the enumerated ones (a simple cycle of m >= 4 relations
// enumerates its m(m - 1) arcs)
struct BlocksW {
    int nb;
    uint64_t cyc;
    uint64_t mask[64];
    uint64_t sub[64];
    uint64_t prefix[65];
    uint64_t eprefix[65];
};

// DFS state of find_blocks64 (local memory for one thread per set, shared
// memory for one lane per warp)
struct DfsScratch {
    uint64_t stk_e[64], desc[64];
    uint8_t disc[64], low[64], parent[64], stk_u[64], vstk[64];
};

__device__ void find_blocks64(uint64_t S, const uint64_t *adj, BlocksW &B, DfsScratch &D) {
    uint8_t *disc = D.disc, *low = D.low, *parent = D.parent, *stk_u = D.stk_u, *vstk = D.vstk;
    uint64_t *stk_e = D.stk_e, *desc = D.desc;
    int sp = 0, vsp = 0, t = 0;
    uint64_t visited = 0;
    B.nb = 0;
    B.cyc = 0;
    uint64_t total = 0, etotal = 0;
    const int root = lowest_idx64(S);
    visited |= 1ull << root;
    disc[root] = (uint8_t)t++;
    low[root] = 255;
    parent[root] = 255;
    desc[root] = 1ull << root;
    vstk[vsp++] = (uint8_t)root;
    stk_u[sp] = (uint8_t)root;
    stk_e[sp] = adj[root] & S;
    sp++;
    while (sp > 0) {
        const int u = stk_u[sp - 1];
        const uint64_t e = stk_e[sp - 1];
        if (e == 0) {
            sp--;
            if (sp > 0) {
                const int p = stk_u[sp - 1];
                if (low[u] >= disc[p]) {
                    uint64_t blk = 1ull << p;
                    int w;
                    do {
                        w = vstk[--vsp];
                        blk |= 1ull << w;
                    } while (w != u);
                    const int m = __popcll(blk);
                    bool cycle = m >= 4;
                    for (uint64_t x = blk; cycle && x; x &= x - 1ull) cycle = __popcll(adj[lowest_idx64(x)] & blk) == 2;
                    B.prefix[B.nb] = total;
                    B.eprefix[B.nb] = etotal;
                    if (cycle) B.cyc |= 1ull << B.nb;
                    B.sub[B.nb] = desc[u];
                    B.mask[B.nb++] = blk;
                    // m <= 63 (at most 63 relations), and the blocks' sizes minus one
                    // sum to |S| - 1, so both totals stay below 2^63
                    total += (1ull << m) - 2ull;
                    etotal += cycle ? (uint64_t)m * (uint64_t)(m - 1) : ((1ull << m) - 2ull);
                }
                if (low[u] < low[p]) low[p] = low[u];
                desc[p] |= desc[u];
                stk_e[sp - 1] &= ~(1ull << u);
            }
            continue;
        }
        const int v = lowest_idx64(e);
        if (!((visited >> v) & 1ull)) {
            visited |= 1ull << v;
            parent[v] = (uint8_t)u;
            disc[v] = (uint8_t)t++;
            low[v] = 255;
            desc[v] = 1ull << v;
            vstk[vsp++] = (uint8_t)v;
            stk_u[sp] = (uint8_t)v;
            stk_e[sp] = adj[v] & S;
            sp++;
        } else {
            if (parent[u] != v && disc[v] < disc[u]) {
                if (disc[v] < low[u]) low[u] = disc[v];
            }
            stk_e[sp - 1] = e & ~(1ull << v);
        }
    }
    B.prefix[B.nb] = total;
    B.eprefix[B.nb] = etotal;
}

// prefix masks of a cycle block's walk: from the block's lowest relation
// towards its lower neighbour, pre[i] holds the first i relations of the walk
// (pre[0] = 0 .. pre[m] = the block)
__device__ void cycle_walk64(uint64_t blk, const uint64_t *adj, uint64_t *pre) {
    const uint32_t m = (uint32_t)__popcll(blk);
    int v = lowest_idx64(blk);
    int prev = 63 - __clzll((long long)(adj[v] & blk));
    pre[0] = 0ull;
    for (uint32_t i = 0; i < m; i++) {
        pre[i + 1] = pre[i] | (1ull << v);
        const int nx = lowest_idx64(adj[v] & blk & ~(1ull << prev));
        prev = v;
        v = nx;
    }
}

// arc j of a cycle of m relations from its walk prefixes: it starts at walk
// position j / (m - 1) and has length j % (m - 1) + 1
__device__ __forceinline__ uint64_t cycle_arc64(const uint64_t *pre, uint32_t m, uint64_t j) {
    const uint64_t s = j / (m - 1u), e = s + j % (m - 1u) + 1u;
    return e <= m ? (pre[e] ^ pre[s]) : ((pre[m] ^ pre[s]) | pre[e - m]);
}

// per-warp shared scratch of k_wide_eval: the set's blocks and the walk
// prefixes of its cycle blocks (the cycle blocks' sizes plus one sum to at
// most 102 for 63 relations), written by lane 0
struct WarpScratch {
    BlocksW B;
    DfsScratch dfs;
    uint64_t pre[128];
    uint8_t pre_off[64];
};
constexpr size_t kEvalSmem = kWideInfoBytes + (kWideBlock / 32) * sizeof(WarpScratch);

// candidate c of S: its two sides and its index in the reference's MPDP order;
// false when the grown sides do not cover S
__device__ bool wide_candidate(uint64_t S, const WarpScratch &ws, const uint64_t *adj, uint64_t c, int &b, uint64_t &L,
                               uint64_t &R, uint64_t &key) {
    const BlocksW &B = ws.B;
    while (b + 1 < B.nb && B.eprefix[b + 1] <= c) b++;
    const uint64_t blk = B.mask[b];
    const uint64_t j = c - B.eprefix[b];
    if (__popcll(blk) == 2) {
        const uint64_t lo = lowest64(blk);
        const uint64_t lb = (j == 0u) ? lo : (blk ^ lo);
        const uint64_t sub = B.sub[b];
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
    uint64_t lb;
    if ((B.cyc >> b) & 1ull) {
        lb = cycle_arc64(ws.pre + ws.pre_off[b], (uint32_t)__popcll(blk), j);
        key = B.prefix[b] + pext64(lb, blk) - 1ull;
        if (blk == S) {
            L = lb;
            R = S ^ lb;
            return true;
        }
    } else {
        lb = pdep64(j + 1ull, blk);
        key = B.prefix[b] + j;
    }
    const uint64_t rb = blk ^ lb;
    L = grow64(lowest64(lb), S & ~rb, adj);
    R = grow64(lowest64(rb), S & ~lb, adj);
    return (L | R) == S;
}

// gpuqo_row_estimation.cuh:26-88 on 64-bit sets
__device__ float fkselc_of_ec64(const WideInfo &w, int off_fk, uint64_t ec, uint64_t outer, uint64_t inner) {
    for (uint64_t tmp = outer; tmp; tmp &= tmp - 1ull) {
        const uint64_t out_id = lowest64(tmp);
        const int out_idx = __popcll((out_id - 1ull) & ec);
        const uint64_t match = inner & w.fks[off_fk + out_idx];
        if (match) return w.fksel[lowest_idx64(match)];
    }
    return __int_as_float(0x7fffffff);
}

__device__ float ec_selectivity64(const WideInfo &w, int i, uint64_t ec, uint64_t ml, uint64_t mr) {
    const uint32_t off = w.ec_off[i];
    const int off_sels = (int)(off >> 16), off_fks = (int)(off & 0xFFFFu);
    float fk = fkselc_of_ec64(w, off_fks, ec, ml, mr);
    if (!isnan(fk)) return fk;
    fk = fkselc_of_ec64(w, off_fks, ec, mr, ml);
    if (!isnan(fk)) return fk;
    const int size = __popcll(ec);
    int il = __popcll((lowest64(ml) - 1ull) & ec);
    int ir = __popcll((lowest64(mr) - 1ull) & ec);
    if (il > ir) {
        const int t = il;
        il = ir;
        ir = t;
    }
    return w.sels[off_sels + il * size - il * (il + 1) / 2 + (ir - il - 1)];
}

// join_eval_t's general path on 64-bit sets, the classes in class order:
// every class, or (MASKED) only the classes in cmask, which must hold every
// class with a member on each side (the classes of the split edge of a tree
// whose classes all sit on edges, or the intersection of the sides' class
// masks)
template <bool MASKED>
__device__ RelVal join_eval_w(const WideInfo &w, uint64_t L, const RelVal &l, uint64_t R, const RelVal &r,
                              uint64_t cmask = 0ull) {
    auto for_classes = [&](auto &&body) {
        if (MASKED) {
            for (uint64_t m = cmask; m; m &= m - 1ull) body(lowest_idx64(m));
        } else {
            for (int i = 0; i < w.n_ec; i++) body(i);
        }
    };
    const DevHeader &h = w.h;
    const bool inner_single = (R & (R - 1ull)) == 0ull;
    Htsz hz;
    if (r.hz) {
        hz.numbuckets = 1 << ((r.hz >> 1) & 31u);
        hz.numbatches = 1 << (r.hz >> 6);
    } else {
        hz = exec_choose_hash_table_size(r.rows, r.width, h.work_mem);
    }
    const int nbuckets = f2i_x86((float)hz.numbuckets * (float)hz.numbatches);
    float sel = 1.0f, per_tuple = 0.0f, bucketsize = 1.0f, mcvfreq = 1.0f;
    int n_quals = 0;
    bool inner_unique = false, any_index = false;
    for_classes([&](int i) {
        const uint64_t ec = w.ec_relids[i];
        const uint64_t ml = ec & L, mr = ec & R;
        if (!ml || !mr) return;
        const float4 pf = __ldg(w.pair + i);
        if (__float_as_uint(pf.z) != 0u) {
            // a plain class: what the general steps below compute for it
            sel *= (lowest64(ec) & L) ? pf.x : pf.y;
            per_tuple += h.cpu_operator_cost;
            n_quals++;
            if (bucketsize > 0.1f) bucketsize = 0.1f;
            if (mcvfreq > 0.0f) mcvfreq = 0.0f;
            return;
        }
        sel *= ec_selectivity64(w, i, ec, ml, mr);
        per_tuple += h.cpu_operator_cost;
        n_quals++;
        const int off_fks = (int)(w.ec_off[i] & 0xFFFFu);
        bool first = true;
        for (uint64_t m = mr; m; m &= m - 1ull) {
            const uint64_t in_id = lowest64(m);
            const DevVar v = w.vars[off_fks + __popcll((in_id - 1ull) & ec)];
            if (first && inner_single) {
                if ((v.flags & 1u) && (v.flags & 2u)) inner_unique = true;
                if (v.flags & 1u) any_index = true;
            }
            first = false;
            const float this_bs = bucketsize_one(v, nbuckets);
            if (bucketsize > this_bs) bucketsize = this_bs;
            if (mcvfreq > v.mcvfreq) mcvfreq = v.mcvfreq;
        }
    });
    RelVal out;
    const float rows = sel * l.rows * r.rows;
    out.rows = rows > 1.0f ? roundf(rows) : 1.0f;
    out.width = l.width + r.width;
    Extra extra;
    extra.inner_unique = inner_unique;
    extra.indexed_join_quals = false;
    extra.joinrows = out.rows;
    extra.outer_match_frac = inner_unique ? out.rows / (l.rows * r.rows) : 0.0f;
    extra.match_count = r.rows;
    float min_s, min_t, s, t;
    cost_nestloop(h, l, r.rows, r.startup, r.total, extra, per_tuple, min_s, min_t);
    if (h.enable_hashjoin) {
        cost_hashjoin(h, l, r, extra, n_quals, per_tuple, hz, bucketsize, mcvfreq, s, t);
        if (t < min_t) {
            min_s = s;
            min_t = t;
        }
    }
    if (any_index && !((w.composite >> lowest_idx64(R)) & 1ull)) {
        extra.indexed_join_quals = true;
        for_classes([&](int i) {
            const uint64_t ec = w.ec_relids[i];
            const uint64_t ml = ec & L, mr = ec & R;
            if (!ml || !mr) return;
            const int off_fks = (int)(w.ec_off[i] & 0xFFFFu);
            const DevVar v = w.vars[off_fks + __popcll((lowest64(mr) - 1ull) & ec)];
            if (!(v.flags & 1u)) return;
            cost_nestloop(h, l, v.idx_rows, v.idx_startup, v.idx_total, extra, per_tuple, s, t);
            if (t < min_t) {
                min_s = s;
                min_t = t;
            }
        });
    }
    out.startup = min_s;
    out.total = min_t;
    return out;
}

// open-addressing table from a connected set to its memo slot
struct WideTable {
    unsigned long long *keys;          // [cap], 0 = empty (no set is empty)
    uint32_t *slot;                    // [cap]
    uint32_t cap_log2;
};

__device__ __forceinline__ uint32_t wide_hash(uint64_t key, uint32_t cap_log2) {
    return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> (64 - cap_log2));
}

// one set into the table with its slot (linear probing; the table is never
// more than half full, so a free slot is always found)
__device__ __forceinline__ void wide_insert_one(const WideTable &t, unsigned long long key, uint32_t slot,
                                                unsigned *err) {
    const uint32_t cap = 1u << t.cap_log2;
    uint32_t pos = wide_hash(key, t.cap_log2);
    for (uint32_t probe = 0; probe < cap; probe++, pos = (pos + 1u) & (cap - 1u)) {
        const unsigned long long old = atomicCAS(t.keys + pos, 0ull, key);
        if (old == 0ull || old == key) {
            t.slot[pos] = slot;
            return;
        }
    }
    atomicExch(err, 1u);
}

// sets[first .. first + count) into the table, each with its index as slot
__global__ void k_wide_insert(WideTable t, const unsigned long long *__restrict__ sets, uint32_t first,
                              uint32_t count, unsigned *__restrict__ err) {
    for (uint32_t i = first + blockIdx.x * blockDim.x + threadIdx.x; i < first + count;
         i += gridDim.x * blockDim.x)
        wide_insert_one(t, sets[i], i, err);
}

__device__ __forceinline__ uint32_t wide_lookup(const WideTable &t, uint64_t key, unsigned *err) {
    const uint32_t cap = 1u << t.cap_log2;
    uint32_t pos = wide_hash(key, t.cap_log2);
    for (uint32_t probe = 0; probe < cap; probe++, pos = (pos + 1u) & (cap - 1u)) {
        const unsigned long long k = __ldg(t.keys + pos);
        if (k == key) return __ldg(t.slot + pos);
        if (k == 0ull) break;
    }
    atomicExch(err, 2u);                  // a side that is not a connected set: cannot happen
    return 0u;
}

__device__ __forceinline__ RelVal wide_rel(const float4 *memo, uint32_t slot, uint32_t packed) {
    return unpack_rel(__ldcg(memo + slot), packed);
}

// one warp per connected set of level k (sets[first .. first + count))
__global__ void __launch_bounds__(kWideBlock) k_wide_eval(const WideInfo *__restrict__ wi, WideTable t,
                                                          const unsigned long long *__restrict__ sets, uint32_t first,
                                                          uint32_t count, int index_order, float4 *__restrict__ memo,
                                                          unsigned long long *__restrict__ memo_left,
                                                          unsigned long long *__restrict__ pairs_out,
                                                          unsigned *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char wsm[];
    WideInfo &w = *reinterpret_cast<WideInfo *>(wsm);
    for (uint32_t x = threadIdx.x; x < (uint32_t)(sizeof(WideInfo) / 4); x += blockDim.x)
        reinterpret_cast<uint32_t *>(wsm)[x] = reinterpret_cast<const uint32_t *>(wi)[x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    WarpScratch &ws = reinterpret_cast<WarpScratch *>(wsm + kWideInfoBytes)[threadIdx.x >> 5];
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long pairs = 0;
    for (uint32_t i = gwarp; i < count; i += nwarps) {
        const uint64_t S = sets[first + i];
        __syncwarp();   // every lane is done with the previous set's scratch
        if (lane == 0) {
            find_blocks64(S, w.adj, ws.B, ws.dfs);
            uint32_t off = 0;
            for (int b = 0; b < ws.B.nb; b++) {
                ws.pre_off[b] = (uint8_t)off;
                if ((ws.B.cyc >> b) & 1ull) {
                    cycle_walk64(ws.B.mask[b], w.adj, ws.pre + off);
                    off += (uint32_t)__popcll(ws.B.mask[b]) + 1u;
                }
            }
        }
        __syncwarp();
        const BlocksW &B = ws.B;
        const uint64_t P = B.eprefix[B.nb];
        if (P > kWideMaxCandidates) {   // a dense block: far beyond what an exact DP at this size can afford
            if (lane == 0) atomicExch(err, 3u);
            continue;
        }
        // lane best: (ordered cost, index) lexicographic; first valid
        // candidate (index, NaN) for the reference's NaN rule
        uint32_t best_c = kFullW;
        uint64_t best_k = ~0ull, first_k = ~0ull;
        bool first_nan = false;
        RelVal best_v, nan_v;
        uint64_t best_l = 0, nan_l = 0;
        int b = 0;
        for (uint64_t c = (uint64_t)lane; c < P; c += 32u) {
            uint64_t L, R, key;
            if (!wide_candidate(S, ws, w.adj, c, b, L, R, key)) continue;
            if (index_order) key = dpsub_index64(L, S);
            const RelVal l = wide_rel(memo, wide_lookup(t, L, err), w.h.hz_packed);
            const RelVal r = wide_rel(memo, wide_lookup(t, R, err), w.h.hz_packed);
            RelVal out;
            if (w.rel_masked) {
                uint64_t cl = 0ull, cr = 0ull;
                for (uint64_t x = L; x; x &= x - 1ull) cl |= w.rel_cls[lowest_idx64(x)];
                for (uint64_t x = R; x; x &= x - 1ull) cr |= w.rel_cls[lowest_idx64(x)];
                out = join_eval_w<true>(w, L, l, R, r, cl & cr);
            } else {
                out = join_eval_w<false>(w, L, l, R, r);
            }
            const bool nan = isnan(out.total);
            pairs++;
            if (key < first_k) {
                first_k = key;
                first_nan = nan;
                if (nan) {
                    nan_v = out;
                    nan_l = L;
                }
            }
            if (!nan) {
                const uint32_t oc = ord_float(out.total);
                if (oc < best_c || (oc == best_c && key < best_k)) {
                    best_c = oc;
                    best_k = key;
                    best_v = out;
                    best_l = L;
                }
            }
        }
        // warp: minimum cost, then minimum index among it; first candidate
        const uint32_t mc = __reduce_min_sync(kFullW, best_c);
        const uint64_t kc = (best_c == mc) ? best_k : ~0ull;
        const uint32_t kh = __reduce_min_sync(kFullW, (uint32_t)(kc >> 32));
        const uint32_t kl = __reduce_min_sync(kFullW, (uint32_t)(kc >> 32) == kh ? (uint32_t)kc : kFullW);
        const uint64_t mk = ((uint64_t)kh << 32) | kl;
        const uint32_t fh = __reduce_min_sync(kFullW, (uint32_t)(first_k >> 32));
        const uint32_t fl = __reduce_min_sync(kFullW, (uint32_t)(first_k >> 32) == fh ? (uint32_t)first_k : kFullW);
        const uint64_t mf = ((uint64_t)fh << 32) | fl;
        const bool nan_first = first_k == mf && first_nan && mf != ~0ull;
        const unsigned nm = __ballot_sync(kFullW, nan_first);
        const uint32_t slot = (lane == 0) ? wide_lookup(t, S, err) : 0u;
        const uint32_t sslot = __shfl_sync(kFullW, slot, 0);
        const RelVal *wv = nullptr;
        uint64_t wl = 0;
        if (nm) {
            if (nan_first) {
                wv = &nan_v;
                wl = nan_l;
            }
        } else if (best_c == mc && best_k == mk && mc != kFullW) {
            wv = &best_v;
            wl = best_l;
        }
        if (wv) {
            memo[sslot] = make_float4(wv->rows, wv->startup, wv->total,
                                      __uint_as_float(memo_width_word(w.h, wv->rows, wv->width)));
            memo_left[sslot] = wl;
        }
    }
    for (int off = 16; off >= 1; off >>= 1) pairs += __shfl_xor_sync(kFullW, pairs, off);
    if (lane == 0 && pairs) atomicAdd(pairs_out, pairs);
}

// candidate splits of every set of two or more relations, summed: the work
// bound checked before the levels (a set above kWideMaxCandidates counts
// beyond kWideMaxTotal on its own)
__global__ void k_wide_work(const WideInfo *__restrict__ wi, const unsigned long long *__restrict__ sets,
                            uint32_t count, unsigned long long *__restrict__ total) {
    const WideInfo &w = *wi;
    BlocksW B;
    DfsScratch D;
    unsigned long long acc = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint64_t S = sets[i];
        if (__popcll(S) < 2) continue;
        find_blocks64(S, w.adj, B, D);
        const uint64_t P = B.eprefix[B.nb];
        acc += P > kWideMaxCandidates ? kWideMaxTotal + 1u : P;   // one such set refuses the DP
    }
    for (int off = 16; off >= 1; off >>= 1) acc += __shfl_xor_sync(kFullW, acc, off);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(total, acc);
}

__global__ void k_wide_base(const WideInfo *__restrict__ wi, WideTable t, float4 *__restrict__ memo,
                            unsigned long long *__restrict__ memo_left, unsigned *__restrict__ err) {
    const WideInfo &w = *wi;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.n) return;
    // gpuqo_cpu_sequential.cu:80-92: base relation memo entries
    const uint32_t s = wide_lookup(t, 1ull << i, err);
    memo[s] = make_float4(w.rows[i], w.startup[i], w.total[i],
                          __uint_as_float(memo_width_word(w.h, w.rows[i], w.width[i])));
    memo_left[s] = 0ull;
}

// ---------------------------------------------------------------------------
// tree-shaped query graphs: no block search
// ---------------------------------------------------------------------------
// Per-root tables of a tree-shaped graph, row r for the preorder from r with
// children in increasing index order (the DFS order of the reference's block
// search): sub = the relation's subtree, before = the relations ahead of it,
// anc = its ancestors, par = its parent.  Every connected set S is a subtree
// rooted at r = lowest(S); its blocks are its edges, each emitted when the DFS
// returns from the child end c, so the block of edge (par c, c) is number
//     post = |S & before[c]| - |S & anc[c]| + |S & sub[c]| - 1
// and its two candidates (the side holding the lower end first) have the
// reference's indices 2 post and 2 post + 1.
struct WideTree {
    const unsigned long long *sub, *before, *anc;   // [n * n]
    const uint8_t *par;                             // [n * n]
};

__device__ __forceinline__ int nth_bit64(uint64_t x, int e) {   // the e-th set bit of x, from 0
    const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    const int c = __popc(lo);
    return e < c ? (int)__fns(lo, 0u, e + 1) : 32 + (int)__fns(hi, 0u, e - c + 1);
}

// level k + 1 of a tree-shaped graph from level k: adding a neighbour u to a
// connected S makes u a leaf of T = S + u, and T is emitted only from the S
// whose u is T's largest leaf, so every connected set appears once.  Output
// at sets[out_first + atomic index], entered into the table with that slot;
// an index at or beyond out_count (which the host counted exactly) raises
// err 4 instead of writing.
__global__ void __launch_bounds__(256) k_wide_tree_enum(const WideInfo *__restrict__ wi, WideTable t,
                                                        unsigned long long *__restrict__ sets, uint32_t first,
                                                        uint32_t count, uint32_t out_first, uint32_t out_count,
                                                        unsigned *__restrict__ out_n, unsigned *__restrict__ err) {
    __shared__ unsigned long long adj[64];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) adj[i] = wi->adj[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t rounds = (count + stride - 1u) / stride;
    for (uint32_t rd = 0; rd < rounds; rd++) {
        const uint32_t i = rd * stride + blockIdx.x * blockDim.x + threadIdx.x;
        uint64_t S = 0ull, N = 0ull, leaves = 0ull;
        if (i < count) {
            S = sets[first + i];
            for (uint64_t x = S; x; x &= x - 1ull) {
                const int v = lowest_idx64(x);
                const uint64_t a = adj[v];
                N |= a;
                if (__popcll(a & S) == 1) leaves |= 1ull << v;
            }
            N &= ~S;
        }
        const bool single = (S & (S - 1ull)) == 0ull;
        const int deg = __popcll(N);
        const int maxdeg = (int)__reduce_max_sync(kFullW, (uint32_t)deg);
        for (int j = 0; j < maxdeg; j++) {
            bool ok = false;
            uint64_t T = 0ull;
            if (j < deg) {
                const uint64_t bu = lowest64(N);
                N ^= bu;
                T = S | bu;
                const uint64_t p = adj[lowest_idx64(bu)] & S;          // u's only neighbour in S
                const uint64_t others = single ? S : (leaves & ~p);    // T's other leaves
                ok = others < bu;                                       // u is T's largest leaf
            }
            const unsigned m = __ballot_sync(kFullW, ok);
            if (m) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(out_n, (unsigned)__popc(m));
                base = __shfl_sync(kFullW, base, 0);
                if (ok) {
                    const uint32_t idx = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
                    if (idx < out_count) {
                        sets[out_first + idx] = T;
                        wide_insert_one(t, T, out_first + idx, err);
                    } else {
                        atomicExch(err, 4u);
                    }
                }
            }
        }
    }
}

// level k of a tree-shaped graph: groups of G lanes (a power of two) per set,
// a lane per edge (two when k - 1 > 32), both orientations of each edge
__global__ void __launch_bounds__(kWideBlock) k_wide_eval_tree(const WideInfo *__restrict__ wi, WideTable t,
                                                               WideTree tt, const unsigned long long *__restrict__ sets,
                                                               uint32_t first, uint32_t count, int k, int G,
                                                               int index_order, float4 *__restrict__ memo,
                                                               unsigned long long *__restrict__ memo_left,
                                                               unsigned long long *__restrict__ pairs_out,
                                                               unsigned *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char wsm[];
    WideInfo &w = *reinterpret_cast<WideInfo *>(wsm);
    for (uint32_t x = threadIdx.x; x < (uint32_t)(sizeof(WideInfo) / 4); x += blockDim.x)
        reinterpret_cast<uint32_t *>(wsm)[x] = reinterpret_cast<const uint32_t *>(wi)[x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t gpw = 32u / (uint32_t)G;
    const int grp = lane / G, gl = lane % G;
    const uint32_t group_mask = (G == 32) ? kFullW : (((1u << G) - 1u) << (grp * G));
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int n = w.n;
    const uint32_t E = (uint32_t)(k - 1);
    unsigned long long pairs = 0;
    for (uint32_t i0 = gwarp * gpw; i0 < count; i0 += nwarps * gpw) {
        const uint32_t i = i0 + (uint32_t)grp;
        const uint64_t S = (i < count) ? sets[first + i] : 0ull;
        // a listed set has k relations among the n (anything else is an
        // enumeration fault: reported, never indexed with)
        const bool has = i < count && __popcll(S) == k && (S >> n) == 0ull;
        if (i < count && !has && gl == 0) atomicExch(err, 5u);
        const int r = has ? lowest_idx64(S) : 0;
        const uint64_t Sn = S & ~(1ull << r);
        uint32_t best_c = kFullW;
        uint64_t best_k = ~0ull, first_k = ~0ull, best_l = 0ull, nan_l = 0ull;
        bool first_nan = false;
        RelVal best_v, nan_v;
        best_v.rows = best_v.startup = best_v.total = 0.0f;
        best_v.width = 0;
        best_v.hz = 0u;
        nan_v = best_v;
        auto update = [&](uint64_t key, uint64_t L, const RelVal &out) {
            const bool nan = isnan(out.total);
            if (key < first_k) {
                first_k = key;
                first_nan = nan;
                if (nan) {
                    nan_v = out;
                    nan_l = L;
                }
            }
            if (!nan) {
                const uint32_t oc = ord_float(out.total);
                if (oc < best_c || (oc == best_c && key < best_k)) {
                    best_c = oc;
                    best_k = key;
                    best_v = out;
                    best_l = L;
                }
            }
        };
        for (uint32_t e = (uint32_t)gl; has && e < E; e += (uint32_t)G) {
            const int v = nth_bit64(Sn, (int)e);
            const int p = tt.par[r * n + v];
            const uint64_t comp = S & __ldg(tt.sub + r * n + v);
            const uint64_t L0 = (v < p) ? comp : (S ^ comp);     // the side holding the edge's lower end
            const uint64_t R0 = S ^ L0;
            uint64_t k0, k1;
            if (index_order) {
                k0 = dpsub_index64(L0, S);
                k1 = dpsub_index64(R0, S);
            } else {
                const uint64_t post = (uint64_t)(__popcll(S & __ldg(tt.before + r * n + v)) -
                                                 __popcll(S & __ldg(tt.anc + r * n + v)) + __popcll(comp) - 1);
                k0 = 2ull * post;
                k1 = k0 + 1ull;
            }
            const RelVal lv = wide_rel(memo, wide_lookup(t, L0, err), w.h.hz_packed);
            const RelVal rv = wide_rel(memo, wide_lookup(t, R0, err), w.h.hz_packed);
            if (w.edge_masked) {
                const int child0 = ((__ldg(tt.anc + v) >> p) & 1ull) ? v : p;   // w.r.t. relation 0
                const uint64_t cm = w.edge_cls[child0];
                update(k0, L0, join_eval_w<true>(w, L0, lv, R0, rv, cm));
                update(k1, R0, join_eval_w<true>(w, R0, rv, L0, lv, cm));
            } else if (w.rel_masked) {
                uint64_t cl = 0ull, cr = 0ull;
                for (uint64_t x = L0; x; x &= x - 1ull) cl |= w.rel_cls[lowest_idx64(x)];
                for (uint64_t x = R0; x; x &= x - 1ull) cr |= w.rel_cls[lowest_idx64(x)];
                update(k0, L0, join_eval_w<true>(w, L0, lv, R0, rv, cl & cr));
                update(k1, R0, join_eval_w<true>(w, R0, rv, L0, lv, cl & cr));
            } else {
                update(k0, L0, join_eval_w<false>(w, L0, lv, R0, rv));
                update(k1, R0, join_eval_w<false>(w, R0, rv, L0, lv));
            }
            pairs += 2;
        }
        // group minimum of (cost, index) and of the first index (butterfly
        // within the aligned group; every lane of the warp takes part)
        uint32_t mc = best_c, kh = (uint32_t)(best_k >> 32), kl = (uint32_t)best_k;
        uint32_t fh = (uint32_t)(first_k >> 32), fl = (uint32_t)first_k;
        for (int off = G / 2; off >= 1; off >>= 1) {
            const uint32_t oc = __shfl_xor_sync(kFullW, mc, off);
            const uint32_t oh = __shfl_xor_sync(kFullW, kh, off);
            const uint32_t ol = __shfl_xor_sync(kFullW, kl, off);
            if (oc < mc || (oc == mc && (oh < kh || (oh == kh && ol < kl)))) {
                mc = oc;
                kh = oh;
                kl = ol;
            }
            const uint32_t ofh = __shfl_xor_sync(kFullW, fh, off);
            const uint32_t ofl = __shfl_xor_sync(kFullW, fl, off);
            if (ofh < fh || (ofh == fh && ofl < fl)) {
                fh = ofh;
                fl = ofl;
            }
        }
        const uint64_t mk = ((uint64_t)kh << 32) | kl, mf = ((uint64_t)fh << 32) | fl;
        const bool nan_first = has && first_k == mf && first_nan && mf != ~0ull;
        const unsigned nm = __ballot_sync(kFullW, nan_first) & group_mask;
        const RelVal *wv = nullptr;
        uint64_t wl = 0ull;
        if (has) {
            if (nm) {
                if (nan_first) {
                    wv = &nan_v;
                    wl = nan_l;
                }
            } else if (best_c == mc && best_k == mk && mc != kFullW) {
                wv = &best_v;
                wl = best_l;
            }
        }
        if (wv) {
            const uint32_t slot = wide_lookup(t, S, err);
            memo[slot] = make_float4(wv->rows, wv->startup, wv->total,
                                     __uint_as_float(memo_width_word(w.h, wv->rows, wv->width)));
            memo_left[slot] = wl;
        }
    }
    for (int off = 16; off >= 1; off >>= 1) pairs += __shfl_xor_sync(kFullW, pairs, off);
    if (lane == 0 && pairs) atomicAdd(pairs_out, pairs);
}

// level k + 1 of any graph from level k, listed on the device: every
// extension of a set by one neighbour is offered to the table, and the thread
// whose atomicCAS claims the key appends the set (so each connected set is
// listed once, whichever of its subsets offered it first).  Indices from
// out_first on; an index at or beyond out_cap raises err 6 instead of writing.
__global__ void __launch_bounds__(256) k_wide_list_ext(const WideInfo *__restrict__ wi, WideTable t,
                                                       unsigned long long *__restrict__ sets, uint32_t first,
                                                       uint32_t count, uint32_t out_first, uint32_t out_cap,
                                                       unsigned *__restrict__ out_n, unsigned *__restrict__ err) {
    namespace cg = cooperative_groups;
    __shared__ unsigned long long adj[64];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) adj[i] = wi->adj[i];
    __syncthreads();
    const uint32_t cap = 1u << t.cap_log2;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint64_t S = sets[first + i];
        uint64_t N = 0ull;
        for (uint64_t x = S; x; x &= x - 1ull) N |= adj[lowest_idx64(x)];
        N &= ~S;
        for (; N; N &= N - 1ull) {
            const unsigned long long T = S | lowest64(N);
            uint32_t pos = wide_hash(T, t.cap_log2);
            bool done = false;
            for (uint32_t probe = 0; probe < cap && !done; probe++) {
                const unsigned long long old = atomicCAS(t.keys + pos, 0ull, T);
                if (old == 0ull) {
                    // claimed: append (one counter update per group of claimers)
                    cg::coalesced_group g = cg::coalesced_threads();
                    unsigned base = 0;
                    if (g.thread_rank() == 0) base = atomicAdd(out_n, g.size());
                    base = g.shfl(base, 0);
                    const uint32_t idx = out_first + base + g.thread_rank();
                    if (idx < out_cap) {
                        sets[idx] = T;
                        t.slot[pos] = idx;
                    } else {
                        atomicExch(err, 6u);
                    }
                    done = true;
                } else if (old == T) {
                    done = true;   // listed already
                } else {
                    pos = (pos + 1u) & (cap - 1u);
                }
            }
            if (!done) atomicExch(err, 1u);
        }
    }
}

// the plan, walked from the full set by one thread (at most 2n - 1 nodes)
__global__ void k_wide_extract(WideTable t, const float4 *__restrict__ memo,
                               const unsigned long long *__restrict__ memo_left, uint64_t full, int n,
                               uint32_t wmask, TreeNode *__restrict__ out, int *__restrict__ n_out,
                               unsigned *__restrict__ err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint64_t st_set[128];
    int st_parent[128], st_side[128];
    int sp = 0, cnt = 0;
    st_set[sp] = full;
    st_parent[sp] = -1;
    st_side[sp] = 0;
    sp++;
    while (sp > 0 && cnt < 2 * n - 1) {
        sp--;
        const uint64_t s = st_set[sp];
        const int parent = st_parent[sp], side = st_side[sp];
        const uint32_t slot = wide_lookup(t, s, err);
        const float4 v = __ldcg(memo + slot);
        TreeNode nd;
        nd.set = s;
        nd.left = -1;
        nd.right = -1;
        nd.rows = v.x;
        nd.startup = v.y;
        nd.total = v.z;
        nd.width = (int32_t)(__float_as_uint(v.w) & wmask);
        const int me = cnt++;
        out[me] = nd;
        if (parent >= 0) {
            if (side == 0) out[parent].left = me;
            else out[parent].right = me;
        }
        const uint64_t l = __ldcg(memo_left + slot) & s;
        if (__popcll(s) > 1 && l != 0ull && l != s && sp + 2 <= 128) {
            st_set[sp] = s ^ l;
            st_parent[sp] = me;
            st_side[sp] = 1;
            sp++;
            st_set[sp] = l;
            st_parent[sp] = me;
            st_side[sp] = 0;
            sp++;
        }
    }
    *n_out = cnt;
}

#define CKW(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            cudaGetLastError();                                                           \
            rc = (e_ == cudaErrorMemoryAllocation) ? GPUQO_B200_ERR_NOMEM : GPUQO_B200_ERR_CUDA; \
            goto done;                                                                    \
        }                                                                                 \
    } while (0)

}  // namespace

uint64_t wide_set_capacity() { return 1ull << 25; }

// Whether every biconnected block of the (connected) graph is a bridge or a
// simple cycle: a block of m relations holding at most m edges.  Blocks by
// Hopcroft-Tarjan on the host (recursive, at most 63 relations deep).
static bool is_cactus(const std::vector<uint64_t> &adj) {
    const int n = (int)adj.size();
    std::vector<int> disc(n, -1), low(n, 0), vstack;
    int t = 0;
    bool ok = true;
    std::function<void(int, int)> dfs = [&](int u, int parent) {
        disc[u] = low[u] = t++;
        vstack.push_back(u);
        for (uint64_t x = adj[u]; x && ok; x &= x - 1ull) {
            const int v = __builtin_ctzll(x);
            if (disc[v] < 0) {
                dfs(v, u);
                low[u] = std::min(low[u], low[v]);
                if (low[v] >= disc[u]) {
                    uint64_t blk = 1ull << u;
                    int w;
                    do {
                        w = vstack.back();
                        vstack.pop_back();
                        blk |= 1ull << w;
                    } while (w != v);
                    int m = 0, deg2 = 0;
                    for (uint64_t y = blk; y; y &= y - 1ull) {
                        m++;
                        deg2 += __builtin_popcountll(adj[__builtin_ctzll(y)] & blk);
                    }
                    if (deg2 / 2 > m) ok = false;
                }
            } else if (v != parent) {
                low[u] = std::min(low[u], disc[v]);
            }
        }
    };
    if (n > 0) dfs(0, -1);
    return ok;
}

// Device state of the sparse DP, kept per device across calls: grow-only
// buffers, a stream and two events.  One sparse DP at a time per device
// (its mutex); the buffers stay allocated for the next call, as the dense
// engine's arenas do.
struct WideArena {
    std::mutex mu;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void *buf[24] = {};
    size_t cap[24] = {};
};
static WideArena g_wide_arena[64];

static cudaError_t arena_get(WideArena &a, int idx, size_t bytes, void **out) {
    if (a.cap[idx] < bytes) {
        if (a.buf[idx]) cudaFree(a.buf[idx]);
        a.buf[idx] = nullptr;
        a.cap[idx] = 0;
        const cudaError_t e = cudaMalloc(&a.buf[idx], bytes);
        if (e != cudaSuccess) {
            a.buf[idx] = nullptr;
            return e;
        }
        a.cap[idx] = bytes;
    }
    *out = a.buf[idx];
    return cudaSuccess;
}

// Connected sets of a tree per size (index 1..n), counted without listing
// them: g_v(x) = x * prod over v's children c of (1 + g_c(x)) counts the sets
// whose relation nearest the root is v; doubles, exact below 2^53.
static std::vector<double> tree_level_counts(const std::vector<uint64_t> &adj) {
    const int n = (int)adj.size();
    std::vector<int> order(1, 0), parent(n, -1);
    std::vector<bool> seen(n, false);
    seen[0] = true;
    for (size_t q = 0; q < order.size(); q++) {
        const int u = order[q];
        for (uint64_t x = adj[u]; x; x &= x - 1ull) {
            const int v = __builtin_ctzll(x);
            if (!seen[v]) {
                seen[v] = true;
                parent[v] = u;
                order.push_back(v);
            }
        }
    }
    std::vector<std::vector<double>> g(n, std::vector<double>(n + 1, 0.0));
    std::vector<double> out(n + 1, 0.0);
    for (int q = n - 1; q >= 0; q--) {
        const int v = order[q];
        std::vector<double> acc(n + 1, 0.0);
        acc[1] = 1.0;
        for (uint64_t x = adj[v]; x; x &= x - 1ull) {
            const int c = __builtin_ctzll(x);
            if (parent[c] != v) continue;
            std::vector<double> nx(n + 1, 0.0);
            for (int a = 1; a <= n; a++) {
                if (acc[a] == 0.0) continue;
                nx[a] += acc[a];
                for (int b = 1; a + b <= n; b++) nx[a + b] += acc[a] * g[c][b];
            }
            acc.swap(nx);
        }
        g[v] = acc;
        for (int k = 1; k <= n; k++) out[k] += acc[k];
    }
    return out;
}

// per-root tables of a tree (WideTree), rows of n
static void tree_tables(const std::vector<uint64_t> &adj, std::vector<uint64_t> &sub, std::vector<uint64_t> &before,
                        std::vector<uint64_t> &anc, std::vector<uint8_t> &par) {
    const int n = (int)adj.size();
    sub.assign((size_t)n * n, 0ull);
    before.assign((size_t)n * n, 0ull);
    anc.assign((size_t)n * n, 0ull);
    par.assign((size_t)n * n, 255);
    for (int r = 0; r < n; r++) {
        uint64_t *S = &sub[(size_t)r * n], *B = &before[(size_t)r * n], *A = &anc[(size_t)r * n];
        uint8_t *P = &par[(size_t)r * n];
        std::vector<int> stack(1, r), order;
        uint64_t ahead = 0ull;
        while (!stack.empty()) {
            const int u = stack.back();
            stack.pop_back();
            B[u] = ahead;
            ahead |= 1ull << u;
            order.push_back(u);
            uint64_t kids = adj[u] & ~(P[u] == 255 ? 0ull : (1ull << P[u]));
            // pushed from the highest index, so that the lowest is visited first
            while (kids) {
                const int c = 63 - __builtin_clzll(kids);
                kids &= ~(1ull << c);
                P[c] = (uint8_t)u;
                A[c] = A[u] | (1ull << u);
                stack.push_back(c);
            }
        }
        for (int v = 0; v < n; v++) S[v] = 1ull << v;
        for (int q = (int)order.size() - 1; q > 0; q--) S[P[order[q]]] |= S[order[q]];
    }
}

int engine_run_wide(const HostInfo &info, DpMode mode, std::vector<TreeNode> &nodes, EngineStats &st,
                    std::string &err) {
    const int n = info.n;
    if (n < 1 || n > kWideMaxRels) {
        err = "the sparse exact DP takes 1..63 relations";
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    if (mode != kModeMpdp && mode != kModeDpsub) {
        err = "beyond 31 relations the exact DP serves DPsub and MPDP only";
        return GPUQO_B200_ERR_UNSUPPORTED;
    }
    if (info.ec_sels.size() >= 65536 || info.ec_fks.size() >= 65536) {
        err = "too many equivalence-class entries";
        return GPUQO_B200_ERR_ARGS;
    }
    // compact adjacency (relation i = bit i)
    std::vector<uint64_t> adj(n);
    int degree_sum = 0;
    for (int i = 0; i < n; i++) {
        adj[i] = info.edge[i] >> 1;
        degree_sum += __builtin_popcountll(adj[i]);
    }
    const uint64_t full = (n == 64) ? ~0ull : ((1ull << n) - 1ull);
    // Device bytes per set: key + slot at up to 4 table slots per set, the set,
    // its memo entry and its left side; a device-memory budget lowers the cap.
    constexpr uint64_t kBytesPerSet = 4 * 12 + 8 + 16 + 8;
    uint64_t cap_sets = wide_set_capacity();
    bool budget_bound = false;
    if (gpuqo_b200_device_memory_mb > 0) {
        const uint64_t by_budget = ((uint64_t)gpuqo_b200_device_memory_mb << 20) / kBytesPerSet;
        if (by_budget < cap_sets) {
            cap_sets = by_budget;
            budget_bound = true;
        }
    }
    auto too_many = [&]() {
        if (budget_bound) {
            err = "more than " + std::to_string(cap_sets) + " connected sets: beyond gpuqo_b200_device_memory_mb (" +
                  std::to_string(gpuqo_b200_device_memory_mb) + " MB) for the sparse exact DP";
            return GPUQO_B200_ERR_NOMEM;
        }
        err = "more than " + std::to_string(cap_sets) + " connected sets: beyond the sparse memo of the exact DP "
              "(use IDP)";
        return GPUQO_B200_ERR_TOO_LARGE;
    };
    // Connected sets by level.  A tree's are counted on the host and listed
    // on the device level by level (k_wide_tree_enum); other graphs' are
    // listed on the host by extension with one neighbour, deduplicated.
    const bool tree = degree_sum == 2 * (n - 1);
    const uint64_t kHostListMax = gpuqo_b200_sparse_host_list > 0 ? (uint64_t)gpuqo_b200_sparse_host_list : (1ull << 16);
    bool dev_list = false;   // a general graph whose levels the device lists
    std::vector<uint64_t> all;
    std::vector<uint32_t> lvl_off(1, 0);
    if (tree) {
        const std::vector<double> cnt = tree_level_counts(adj);
        double tot = 0.0;
        for (int k = 1; k <= n; k++) tot += cnt[k];
        if (cnt[n] != 1.0) {
            err = "query graph is not connected";
            return GPUQO_B200_ERR_ARGS;
        }
        if (tot > (double)cap_sets) return too_many();
        for (int k = 1; k <= n; k++) lvl_off.push_back(lvl_off.back() + (uint32_t)cnt[k]);
    } else {
        // the host lists up to kHostListMax sets; beyond that the device lists
        // the levels itself (k_wide_list_ext) into arrays of cap_sets entries
        const uint64_t host_max = std::min<uint64_t>(cap_sets, kHostListMax);
        auto over = [&]() -> int {
            if (host_max < cap_sets) {
                dev_list = true;
                return 0;
            }
            return (int)too_many();
        };
        std::vector<uint64_t> cur;
        for (int i = 0; i < n; i++) cur.push_back(1ull << i);
        for (int k = 1; k <= n && !dev_list; k++) {
            if (all.size() + cur.size() > host_max) {
                if (int rc = over()) return rc;
                break;
            }
            all.insert(all.end(), cur.begin(), cur.end());
            lvl_off.push_back((uint32_t)all.size());
            if (k == n) break;
            // level k + 1, deduplicated in a flat open-addressing set (0 is
            // never a set), doubled when half full
            std::vector<uint64_t> table(64, 0ull), next;
            size_t used = 0;
            auto slot_of = [](uint64_t key, size_t mask) {
                return (size_t)((key * 0x9E3779B97F4A7C15ull) >> 32) & mask;
            };
            auto add = [&](uint64_t key) {
                if (2 * (used + 1) > table.size()) {
                    std::vector<uint64_t> bigger(table.size() * 2, 0ull);
                    for (uint64_t kk : table) {
                        if (!kk) continue;
                        size_t j = slot_of(kk, bigger.size() - 1);
                        while (bigger[j]) j = (j + 1) & (bigger.size() - 1);
                        bigger[j] = kk;
                    }
                    table.swap(bigger);
                }
                size_t j = slot_of(key, table.size() - 1);
                while (table[j]) {
                    if (table[j] == key) return;
                    j = (j + 1) & (table.size() - 1);
                }
                table[j] = key;
                used++;
                next.push_back(key);
            };
            for (size_t q = 0; q < cur.size() && !dev_list; q++) {
                const uint64_t S = cur[q];
                uint64_t N = 0;
                for (uint64_t x = S; x; x &= x - 1ull) N |= adj[__builtin_ctzll(x)];
                N &= ~S;
                for (; N && !dev_list; N &= N - 1ull) {
                    add(S | (N & (0ull - N)));
                    if (all.size() + next.size() > host_max)
                        if (int rc = over()) return rc;
                }
            }
            cur.swap(next);
        }
        if (dev_list) {
            all.clear();
            for (int i = 0; i < n; i++) all.push_back(1ull << i);
            lvl_off.assign({0u, (uint32_t)n});
        } else if (all.back() != full) {
            err = "query graph is not connected";
            return GPUQO_B200_ERR_ARGS;
        }
    }
    const bool cactus = tree || is_cactus(adj);
    // entries of the set, memo and left arrays (the listed total, or the cap
    // when the device lists)
    const uint32_t total = dev_list ? (uint32_t)cap_sets : lvl_off[n];
    uint32_t listed = dev_list ? (uint32_t)n : total;
    uint32_t cap_log2 = 1;
    while ((1ull << cap_log2) < 2ull * total) cap_log2++;
    const uint64_t cap = 1ull << cap_log2;
    const size_t n_ec = info.ec_relids.size(), n_sels = info.ec_sels.size(), n_fks = info.ec_fks.size();
    const uint64_t tree_bytes = tree ? (uint64_t)n * n * 25 : 0ull;
    const uint64_t bytes = cap * 12ull + (uint64_t)total * (8 + 16 + 8) + n_ec * 12 + n_sels * 4 + n_fks * 40 +
                           sizeof(WideInfo) + tree_bytes + 64 * sizeof(TreeNode) + 4 * 66 + 64;
    if (gpuqo_b200_device_memory_mb > 0 && bytes > ((uint64_t)gpuqo_b200_device_memory_mb << 20)) {
        err = "the sparse exact DP needs " + std::to_string(bytes >> 20) + " MB of device memory; "
              "gpuqo_b200_device_memory_mb allows " + std::to_string(gpuqo_b200_device_memory_mb);
        return GPUQO_B200_ERR_NOMEM;
    }
    // planner info (host)
    WideInfo hw;
    std::memset(&hw, 0, sizeof(hw));
    hw.n = n;
    hw.n_ec = (int)n_ec;
    hw.h.n = n;
    hw.h.cpu_operator_cost = info.p.cpu_operator_cost;
    hw.h.cpu_tuple_cost = info.p.cpu_tuple_cost;
    hw.h.seq_page_cost = info.p.seq_page_cost;
    hw.h.disable_cost = info.p.disable_cost;
    hw.h.work_mem = info.p.work_mem;
    hw.h.enable_nestloop = info.p.enable_nestloop ? 1 : 0;
    hw.h.enable_hashjoin = info.p.enable_hashjoin ? 1 : 0;
    long long width_sum = 0;
    bool width_ok = true;
    for (int i = 0; i < n; i++) {
        width_sum += info.base[i].width;
        width_ok = width_ok && info.base[i].width >= 0;
        hw.adj[i] = adj[i];
        hw.rows[i] = info.base[i].rows;
        hw.tuples[i] = info.base[i].tuples;
        hw.startup[i] = info.base[i].cost.startup;
        hw.total[i] = info.base[i].cost.total;
        hw.width[i] = info.base[i].width;
        hw.fksel[i] = (float)(1.0 / (double)std::fmax(1.0f, info.base[i].tuples));
        if (info.base[i].composite) hw.composite |= 1ull << i;
    }
    hw.h.hz_packed = (width_ok && width_sum < (1ll << kWidthBits)) ? 1u : 0u;
    std::vector<uint64_t> h_relids(n_ec), h_fks(n_fks);
    std::vector<uint32_t> h_off(n_ec);
    std::vector<DevVar> h_vars(n_fks);
    {
        int off_sels = 0, off_fks = 0;
        for (size_t e = 0; e < n_ec; e++) {
            h_relids[e] = info.ec_relids[e] >> 1;
            h_off[e] = ((uint32_t)off_sels << 16) | (uint32_t)off_fks;
            int j = 0;
            for (uint64_t m = h_relids[e]; m; m &= m - 1ull, j++) {
                const int rel = __builtin_ctzll(m);
                const int f = off_fks + j;
                h_fks[f] = info.ec_fks[f] >> 1;
                const VarInfo &vi = info.ec_vars[f];
                DevVar &dv = h_vars[f];
                std::memset(&dv, 0, sizeof(dv));
                dv.idx_rows = vi.index.rows;
                dv.idx_startup = vi.index.cost.startup;
                dv.idx_total = vi.index.cost.total;
                dv.flags = (vi.index.available ? 1u : 0u) | (vi.index.unique ? 2u : 0u);
                devvar_bucket_terms(dv, vi.stats.stadistinct, vi.stats.stanullfrac, vi.stats.mcvfreq, hw.rows[rel],
                                    hw.tuples[rel]);
            }
            off_sels += j * (j - 1) / 2;
            off_fks += j;
        }
    }
    // the plain-class table (the pair selectivities of gpuqo_row_estimation.cuh
    // :26-88 for a two-member class, both orientations)
    std::vector<float4> h_pair(std::max<size_t>(n_ec, 1), make_float4(0.f, 0.f, 0.f, 0.f));
    for (size_t e = 0; e < n_ec; e++) {
        if (__builtin_popcountll(h_relids[e]) != 2) continue;
        const int off_s = (int)(h_off[e] >> 16), off_f = (int)(h_off[e] & 0xFFFFu);
        const int x = __builtin_ctzll(h_relids[e]), y = 63 - __builtin_clzll(h_relids[e]);
        const bool fk_xy = (h_fks[off_f] >> y) & 1ull;       // member x's key matches y
        const bool fk_yx = (h_fks[off_f + 1] >> x) & 1ull;   // member y's key matches x
        const float sel = info.ec_sels[off_s];
        bool plain = true;
        for (int j = 0; j < 2; j++) {
            const DevVar &dv = h_vars[off_f + j];
            plain = plain && (dv.flags & (1u | kVarMcvRatio)) == 0u && (dv.flags & kVarNoDistinct) != 0u &&
                    dv.mcvfreq == 0.0f;
        }
        float4 &pe = h_pair[e];
        pe.x = fk_xy ? hw.fksel[y] : (fk_yx ? hw.fksel[x] : sel);
        pe.y = fk_yx ? hw.fksel[x] : (fk_xy ? hw.fksel[y] : sel);
        uint32_t flag = plain ? 1u : 0u;
        std::memcpy(&pe.z, &flag, 4);
    }
    if (n_ec <= 64) {
        hw.rel_masked = 1;
        for (size_t e = 0; e < n_ec; e++)
            for (uint64_t m = h_relids[e]; m; m &= m - 1ull) hw.rel_cls[__builtin_ctzll(m)] |= 1ull << e;
    }
    std::vector<uint64_t> t_sub, t_before, t_anc;
    std::vector<uint8_t> t_par;
    if (tree) {
        tree_tables(adj, t_sub, t_before, t_anc, t_par);
        bool masked = n_ec <= 64;
        for (size_t e = 0; masked && e < n_ec; e++) {
            const uint64_t rr = h_relids[e];
            if (__builtin_popcountll(rr) != 2) {
                masked = false;
                break;
            }
            const int a = __builtin_ctzll(rr), b = 63 - __builtin_clzll(rr);
            if (!((adj[a] >> b) & 1ull)) {
                masked = false;   // a class between relations that are not adjacent
                break;
            }
            const int child0 = ((t_anc[(size_t)b] >> a) & 1ull) ? b : a;   // row 0: ancestors w.r.t. relation 0
            hw.edge_cls[child0] |= 1ull << e;
        }
        hw.edge_masked = masked ? 1 : 0;
        if (!masked) std::memset(hw.edge_cls, 0, sizeof(hw.edge_cls));
    }
    std::vector<uint64_t> singles(n);
    for (int i = 0; i < n; i++) singles[i] = 1ull << i;
    int rc = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    WideInfo *d_info = nullptr;
    uint64_t *d_relids = nullptr, *d_fks = nullptr;
    uint32_t *d_off = nullptr, *d_slot = nullptr;
    float *d_sels = nullptr;
    DevVar *d_vars = nullptr;
    unsigned long long *d_keys = nullptr, *d_sets = nullptr, *d_left = nullptr, *d_pairs = nullptr;
    unsigned long long *d_tsub = nullptr, *d_tbefore = nullptr, *d_tanc = nullptr;
    uint8_t *d_tpar = nullptr;
    float4 *d_memo = nullptr, *d_pair = nullptr;
    unsigned *d_err = nullptr;     // [0] error flag, [1 .. n] sets listed per level (trees)
    TreeNode *d_nodes = nullptr;
    int *d_nn = nullptr;
    std::vector<unsigned> h_err(n + 2, 0u);
    unsigned long long h_pairs = 0, h_work = 0;
    int h_nn = 0;
    uint32_t launches = 0;
    float ms = 0.f;
    int sm_count = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (dev < 0 || dev >= 64) {
        err = "device ordinal " + std::to_string(dev) + " beyond the sparse DP's device table";
        return GPUQO_B200_ERR_ARGS;
    }
    WideArena &A = g_wide_arena[dev];
    std::lock_guard<std::mutex> arena_lock(A.mu);
    if (!A.stream) CKW(cudaStreamCreateWithFlags(&A.stream, cudaStreamNonBlocking));
    if (!A.ev0) CKW(cudaEventCreate(&A.ev0));
    if (!A.ev1) CKW(cudaEventCreate(&A.ev1));
    stream = A.stream;
    ev0 = A.ev0;
    ev1 = A.ev1;
#define ARENA(i, ptr, bytes) CKW(arena_get(A, i, (size_t)(bytes), reinterpret_cast<void **>(&(ptr))))
    ARENA(0, d_info, sizeof(WideInfo));
    ARENA(1, d_relids, std::max<size_t>(n_ec, 1) * 8);
    ARENA(2, d_off, std::max<size_t>(n_ec, 1) * 4);
    ARENA(3, d_sels, std::max<size_t>(n_sels, 1) * 4);
    ARENA(4, d_fks, std::max<size_t>(n_fks, 1) * 8);
    ARENA(5, d_vars, std::max<size_t>(n_fks, 1) * sizeof(DevVar));
    ARENA(6, d_pair, h_pair.size() * sizeof(float4));
    ARENA(7, d_keys, cap * 8);
    ARENA(8, d_slot, cap * 4);
    ARENA(9, d_sets, (size_t)total * 8);
    ARENA(10, d_memo, (size_t)total * sizeof(float4));
    ARENA(11, d_left, (size_t)total * 8);
    ARENA(12, d_pairs, 16);   // [0] evaluated pairs, [1] the work bound
    ARENA(13, d_err, (size_t)(n + 2) * 4);
    ARENA(14, d_nodes, 128 * sizeof(TreeNode));
    ARENA(15, d_nn, sizeof(int));
    if (tree) {
        ARENA(16, d_tsub, (size_t)n * n * 8);
        ARENA(17, d_tbefore, (size_t)n * n * 8);
        ARENA(18, d_tanc, (size_t)n * n * 8);
        ARENA(19, d_tpar, (size_t)n * n);
        CKW(cudaMemcpyAsync(d_tsub, t_sub.data(), (size_t)n * n * 8, cudaMemcpyHostToDevice, stream));
        CKW(cudaMemcpyAsync(d_tbefore, t_before.data(), (size_t)n * n * 8, cudaMemcpyHostToDevice, stream));
        CKW(cudaMemcpyAsync(d_tanc, t_anc.data(), (size_t)n * n * 8, cudaMemcpyHostToDevice, stream));
        CKW(cudaMemcpyAsync(d_tpar, t_par.data(), (size_t)n * n, cudaMemcpyHostToDevice, stream));
    }
#undef ARENA
    hw.ec_relids = d_relids;
    hw.ec_off = d_off;
    hw.sels = d_sels;
    hw.fks = d_fks;
    hw.vars = d_vars;
    hw.pair = d_pair;
    CKW(cudaMemcpyAsync(d_info, &hw, sizeof(WideInfo), cudaMemcpyHostToDevice, stream));
    CKW(cudaMemcpyAsync(d_pair, h_pair.data(), h_pair.size() * sizeof(float4), cudaMemcpyHostToDevice, stream));
    if (n_ec) {
        CKW(cudaMemcpyAsync(d_relids, h_relids.data(), n_ec * 8, cudaMemcpyHostToDevice, stream));
        CKW(cudaMemcpyAsync(d_off, h_off.data(), n_ec * 4, cudaMemcpyHostToDevice, stream));
    }
    if (n_sels) CKW(cudaMemcpyAsync(d_sels, info.ec_sels.data(), n_sels * 4, cudaMemcpyHostToDevice, stream));
    if (n_fks) {
        CKW(cudaMemcpyAsync(d_fks, h_fks.data(), n_fks * 8, cudaMemcpyHostToDevice, stream));
        CKW(cudaMemcpyAsync(d_vars, h_vars.data(), n_fks * sizeof(DevVar), cudaMemcpyHostToDevice, stream));
    }
    if (tree) CKW(cudaMemcpyAsync(d_sets, singles.data(), (size_t)n * 8, cudaMemcpyHostToDevice, stream));
    else CKW(cudaMemcpyAsync(d_sets, all.data(), all.size() * 8, cudaMemcpyHostToDevice, stream));
    CKW(cudaMemsetAsync(d_keys, 0, cap * 8, stream));
    CKW(cudaMemsetAsync(d_pairs, 0, 16, stream));
    CKW(cudaMemsetAsync(d_err, 0, (size_t)(n + 2) * 4, stream));
    {
        WideTable t{d_keys, d_slot, cap_log2};
        const int index_order = mode == kModeDpsub ? 1 : 0;
        auto grid_for = [&](uint64_t threads) {
            return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sm_count * 8, (threads + 255) / 256));
        };
        CKW(cudaEventRecord(ev0, stream));
        CKW(cudaFuncSetAttribute(k_wide_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEvalSmem));
        if (tree) {
            // level 1, then per level: list level k + 1 into the table, evaluate it
            const WideTree tt{d_tsub, d_tbefore, d_tanc, d_tpar};
            k_wide_insert<<<1, 64, 0, stream>>>(t, d_sets, 0u, (uint32_t)n, d_err);
            k_wide_base<<<1, 64, 0, stream>>>(d_info, t, d_memo, d_left, d_err);
            launches += 2;
            for (int k = 1; k < n; k++) {
                const uint32_t first = lvl_off[k - 1], count = lvl_off[k] - lvl_off[k - 1];
                const uint32_t nfirst = lvl_off[k], ncount = lvl_off[k + 1] - lvl_off[k];
                k_wide_tree_enum<<<grid_for(count), 256, 0, stream>>>(d_info, t, d_sets, first, count, nfirst,
                                                                     ncount, d_err + k + 1, d_err);
                // lanes per set: as few as keep about two warps' worth of sets
                // per resident warp slot (a lane walks its set's edges one after
                // the other: fewer warp rounds per set), up to one lane per edge
                const int E = k;   // split edges of a (k + 1)-set
                const uint64_t want_lanes = (uint64_t)sm_count * 24u * 32u * 2u;
                int G = 1;
                while (G < E && G < 32 && (uint64_t)ncount * (uint64_t)G < want_lanes) G <<= 1;
                k_wide_eval_tree<<<grid_for((uint64_t)ncount * (uint64_t)G), kWideBlock, kWideInfoBytes, stream>>>(
                    d_info, t, tt, d_sets, nfirst, ncount, k + 1, G, index_order, d_memo, d_left, d_pairs, d_err);
                launches += 2;
                CKW(cudaGetLastError());
            }
        } else if (dev_list) {
            // level 1, then per level: list level k + 1 on the device (the table
            // deduplicates), read its size back, check the work bound (graphs
            // that are not cacti), evaluate it
            k_wide_insert<<<1, 64, 0, stream>>>(t, d_sets, 0u, (uint32_t)n, d_err);
            k_wide_base<<<1, 64, 0, stream>>>(d_info, t, d_memo, d_left, d_err);
            launches += 2;
            uint32_t first = 0, count = (uint32_t)n;
            for (int k = 1; k < n; k++) {
                k_wide_list_ext<<<grid_for(count), 256, 0, stream>>>(d_info, t, d_sets, first, count, listed,
                                                                    total, d_err + k + 1, d_err);
                launches++;
                CKW(cudaGetLastError());
                unsigned got = 0, flag = 0;
                CKW(cudaMemcpyAsync(&got, d_err + k + 1, 4, cudaMemcpyDeviceToHost, stream));
                CKW(cudaMemcpyAsync(&flag, d_err, 4, cudaMemcpyDeviceToHost, stream));
                CKW(cudaStreamSynchronize(stream));
                if (flag == 6u || (uint64_t)listed + got > (uint64_t)total) {
                    rc = too_many();
                    goto done;
                }
                if (flag) {
                    err = "sparse memo table inconsistent while listing";
                    rc = GPUQO_B200_ERR_CUDA;
                    goto done;
                }
                first = listed;
                count = got;
                listed += got;
                if (count == 0) break;
                if (!cactus) {
                    k_wide_work<<<grid_for(count), 256, 0, stream>>>(d_info, d_sets + first, count, d_pairs + 1);
                    launches++;
                    CKW(cudaGetLastError());
                    CKW(cudaMemcpyAsync(&h_work, d_pairs + 1, 8, cudaMemcpyDeviceToHost, stream));
                    CKW(cudaStreamSynchronize(stream));
                    if (h_work > kWideMaxTotal) {
                        err = "the sparse exact DP would evaluate more than " + std::to_string(h_work) +
                              " candidate splits (a large biconnected block that is not a cycle; the bound is 2^35, "
                              "2^24 per set): use IDP";
                        rc = GPUQO_B200_ERR_TOO_LARGE;
                        goto done;
                    }
                }
                k_wide_eval<<<grid_for((uint64_t)count * 32), kWideBlock, kEvalSmem, stream>>>(
                    d_info, t, d_sets, first, count, index_order, d_memo, d_left, d_pairs, d_err);
                launches++;
                CKW(cudaGetLastError());
            }
            if (count != 1u) {
                err = "query graph is not connected";
                rc = GPUQO_B200_ERR_ARGS;
                goto done;
            }
        } else {
            k_wide_insert<<<grid_for(total), 256, 0, stream>>>(t, d_sets, 0u, total, d_err);
            k_wide_base<<<1, 64, 0, stream>>>(d_info, t, d_memo, d_left, d_err);
            launches += 2;
            // refuse before the levels when the DP would evaluate too many splits
            // (a large biconnected block that is not a cycle); a cactus graph
            // cannot: every block of a connected set lies in a block of the graph,
            // so its blocks are bridges and whole cycles, at most 63 * 62 splits
            if (!cactus) {
                k_wide_work<<<grid_for(total), 256, 0, stream>>>(d_info, d_sets, total, d_pairs + 1);
                launches++;
                CKW(cudaGetLastError());
                CKW(cudaMemcpyAsync(&h_work, d_pairs + 1, 8, cudaMemcpyDeviceToHost, stream));
                CKW(cudaStreamSynchronize(stream));
            }
            CKW(cudaGetLastError());
            if (h_work > kWideMaxTotal) {
                err = "the sparse exact DP would evaluate more than " + std::to_string(h_work) +
                      " candidate splits (a large biconnected block that is not a cycle; the bound is 2^35, 2^24 "
                      "per set): use IDP";
                rc = GPUQO_B200_ERR_TOO_LARGE;
                goto done;
            }
            for (int k = 2; k <= n; k++) {
                const uint32_t first = lvl_off[k - 1], count = lvl_off[k] - lvl_off[k - 1];
                if (count == 0) continue;
                launches++;
                k_wide_eval<<<grid_for((uint64_t)count * 32), kWideBlock, kEvalSmem, stream>>>(
                    d_info, t, d_sets, first, count, index_order, d_memo, d_left, d_pairs, d_err);
                CKW(cudaGetLastError());
            }
        }
        k_wide_extract<<<1, 32, 0, stream>>>(t, d_memo, d_left, full, n, hw.h.hz_packed ? kWidthMask : 0xFFFFFFFFu,
                                             d_nodes, d_nn, d_err);
        launches++;
        CKW(cudaGetLastError());
        CKW(cudaEventRecord(ev1, stream));
    }
    nodes.resize(128);
    CKW(cudaMemcpyAsync(nodes.data(), d_nodes, 128 * sizeof(TreeNode), cudaMemcpyDeviceToHost, stream));
    CKW(cudaMemcpyAsync(&h_nn, d_nn, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CKW(cudaMemcpyAsync(h_err.data(), d_err, (size_t)(n + 2) * 4, cudaMemcpyDeviceToHost, stream));
    CKW(cudaMemcpyAsync(&h_pairs, d_pairs, 8, cudaMemcpyDeviceToHost, stream));
    CKW(cudaStreamSynchronize(stream));
    CKW(cudaEventElapsedTime(&ms, ev0, ev1));
    if (h_err[0]) {
        err = h_err[0] == 3 ? "a connected set with more than 2^24 candidate splits (a dense biconnected block): "
                              "beyond the sparse exact DP (use IDP)"
                            : "sparse memo table inconsistent";
        rc = h_err[0] == 3 ? GPUQO_B200_ERR_TOO_LARGE : GPUQO_B200_ERR_CUDA;
        goto done;
    }
    if (tree) {
        for (int k = 2; k <= n; k++) {
            if (h_err[k] != lvl_off[k] - lvl_off[k - 1]) {
                err = "tree enumeration listed " + std::to_string(h_err[k]) + " sets of " + std::to_string(k) +
                      " relations where " + std::to_string(lvl_off[k] - lvl_off[k - 1]) + " exist";
                rc = GPUQO_B200_ERR_CUDA;
                goto done;
            }
        }
    }
    if (h_nn != 2 * n - 1) {
        err = "plan extraction produced " + std::to_string(h_nn) + " nodes";
        rc = GPUQO_B200_ERR_CUDA;
        goto done;
    }
    nodes.resize((size_t)h_nn);
    st.connected_sets += listed - (uint32_t)n;
    st.evaluated_pairs += h_pairs;
    st.memo_bytes = std::max<uint64_t>(st.memo_bytes, bytes);
    st.device_ms += ms;
    st.kernel_launches += launches;
done:
    if (rc) nodes.clear();
    // device buffers, stream and events stay in the device's arena
    return rc;
}

}  // namespace gqb
