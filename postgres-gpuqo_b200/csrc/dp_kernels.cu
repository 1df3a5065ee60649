// dp_kernels.cu - sm_100a kernels of the level-synchronous join-order DP and
// the host engine that sequences them.
//
// Per level k = 2..n (the reference's host loop gpuqo_dpsub_common.cu:295-342):
//   k_filter  - combinadic unrank + Gosper stepping over the C(n,k) candidate
//               sets, connectivity test against the adjacency in shared
//               memory, stream compaction of the connected sets in shared
//               memory (one global atomic per 32 survivors).  Replaces the
//               reference's unrankFilteredDPSubKernel + thrust::remove
//               (gpuqo_dpsub_filtered_kernels.cuh:31-109, gpuqo_dpsub_filtered.cu:120).
//   k_eval    - one warp per connected set: csg-cmp candidates (all subsets,
//               or MPDP biconnected-block candidates), CCC queue so that cost
//               evaluations run warp-full, join cost, warp min-reduction on
//               (cost, enumeration index) and a direct dense-memo write.
//               Replaces evaluateFilteredDPSubKernel + the scratchpad scatter
//               into the hash table (gpuqo_dpsub_filtered_kernels.cuh:152-333,
//               gpuqo_dpsub_common.cu:152-166).
//   k_ovf_*   - sets whose candidate count exceeds one warp's share are split
//               into chunks over all warps; each chunk folds its best into a
//               64-bit atomicMin on (ordered cost << 32 | index); a finalize
//               pass re-derives the winner and writes the memo.
// After the last level k_extract walks the memo back-pointers on the device
// and the host copies one small node array (replaces dpsub_buildQueryTree's
// per-node lookups, gpuqo_query_tree.cuh:47-71).
//
// Tie rule: the reference's CPU engines keep the FIRST strict minimum of
// cost.total in their enumeration order (gpuqo_cpu_common.cuh:202).  Keys are
// (ordered cost, enumeration index), so the lexicographic minimum is that
// element; a NaN cost never replaces, and a NaN first candidate is kept, as
// with the reference's '<' comparisons.
//
// The launch sequence of one query is captured once into a CUDA graph per
// (n, mode, ccc) and replayed; the host never synchronises between levels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "dp_device.cuh"
#include "dp_engine.h"
#include "gpuqo_b200.h"

extern "C" int gpuqo_b200_persistent;
extern "C" int gpuqo_b200_barrier_poll_limit;
extern "C" int gpuqo_b200_device_memory_mb;

namespace gqb {

constexpr int kBlock = 256;
constexpr int kWarpsPerBlock = kBlock / 32;
constexpr uint32_t kFull = 0xFFFFFFFFu;
// candidates per warp above which a set goes to the chunked overflow path
constexpr uint32_t kOvfLimit = 32u * 64u;
// candidates per overflow chunk
constexpr uint32_t kChunk = 32u * 64u;
constexpr int kQueueWords = 64 * 3;    // per-warp CCC queue: 64 x (p, L, R)

// units of chunked work of a set with P candidates: plain DPsub costs a split
// and its mirror together (eval_range_dpsub), so its P candidates are P / 2
// units; MPDP candidates are one unit each
__host__ __device__ __forceinline__ uint32_t ovf_work(int mode, uint32_t P) { return mode == kModeDpsub ? P / 2u : P; }

struct LevelCounters {
    uint32_t n_sets;                   // connected sets found by k_filter
    uint32_t chunk_next;               // overflow work counter
    unsigned long long ovf_packed;     // (n_ovf << 40) | n_chunks
    uint32_t n_fb;                     // sets sent to the exact-order fallback
    uint32_t pad;
};

struct GlobalCounters {
    unsigned long long evaluated_pairs;
};

struct DevArena {
    float4 *memo = nullptr;            // [2^n] rows, startup, total, width bits
    uint32_t *memo_left = nullptr;     // [2^n] left (outer) set of the best join
    uint32_t *sets = nullptr;          // [maxC] connected sets of the current level
    uint32_t *sets2 = nullptr;         // [maxC] second level list (levels alternate)
    uint32_t *seen = nullptr;          // [2^n bits] extension dedup bitmap
    uint32_t *ovf_set = nullptr;       // [maxC]
    uint32_t *ovf_P = nullptr;         // [maxC]
    uint32_t *ovf_off = nullptr;       // [maxC] first chunk id
    unsigned long long *ovf_key = nullptr;   // [maxC]
    unsigned long long *ovf_first = nullptr; // [maxC]
    LevelCounters *lvl = nullptr;      // [33]
    GlobalCounters *glob = nullptr;
    uint32_t *blob = nullptr;          // device planner info
    uint32_t *binom = nullptr;         // [33*33] C(i, j)
    TreeNode *tree = nullptr;          // [64]
    int *tree_n = nullptr;
    unsigned *bar = nullptr;           // grid barrier of the persistent kernel: arrivals, generation, error
    // DPsize only (allocated on its first use)
    uint32_t *pos = nullptr;           // [2^n] place of a set in its level list
    uint32_t *bmask = nullptr;         // [maxC] per set of the previous level: places of its discoveries
    uint32_t *bstart = nullptr;        // [maxC] exclusive prefix of the mask popcounts
    uint32_t *tile_sum = nullptr;      // [maxC / kScanTile + 2]
    unsigned long long *disc = nullptr;   // [maxC] discovery key of each set of the level
    uint32_t *level1 = nullptr;        // [32] the level-1 list (place of each relation)
};

// ---------------------------------------------------------------------------
// k_filter: connected k-subsets of n relations
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t unrank_ksubset(uint64_t r, int n, int k, const uint32_t *binom) {
    // r-th k-subset of {0..n-1} in increasing integer order
    uint32_t s = 0;
    int kk = k;
    for (int pos = n - 1; pos >= 0 && kk > 0; pos--) {
        uint32_t c = binom[pos * 33 + kk];     // kk-subsets of {0..pos-1}
        if (r >= c) {
            s |= 1u << pos;
            r -= c;
            kk--;
        }
    }
    return s;
}

__device__ __forceinline__ uint32_t gosper_next(uint32_t v) {
    uint32_t t = v | (v - 1u);
    return (t + 1u) | (((~t & (0u - ~t)) - 1u) >> __ffs(v));
}

__global__ void __launch_bounds__(kBlock) k_filter(const uint32_t *__restrict__ blob, const uint32_t *__restrict__ binom_g,
                                                   int n, int k, unsigned long long total, uint32_t per_thread,
                                                   uint32_t *__restrict__ out_sets, LevelCounters *__restrict__ lc) {
    __shared__ uint32_t adj[kMaxRels];
    __shared__ uint32_t binom[33 * 33];
    __shared__ uint32_t stage[kWarpsPerBlock][64];
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob);
    for (int i = threadIdx.x; i < kMaxRels; i += blockDim.x) adj[i] = (i < n) ? h->adj[i] : 0u;
    for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) binom[i] = binom_g[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *st = stage[warp];
    uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t r0 = tid * per_thread;
    uint64_t r1 = r0 + per_thread < total ? r0 + per_thread : total;
    uint32_t s = r0 < total ? unrank_ksubset(r0, n, k, binom) : 0u;
    uint32_t cnt = 0;
    for (uint32_t j = 0; j < per_thread; j++) {
        uint64_t r = r0 + j;
        bool has = r < r1;
        bool ok = has && is_connected(s, adj);
        uint32_t m = __ballot_sync(kFull, ok);
        if (ok) st[cnt + __popc(m & ((1u << lane) - 1u))] = s;
        cnt += __popc(m);
        __syncwarp();
        if (cnt >= 32) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&lc->n_sets, 32u);
            base = __shfl_sync(kFull, base, 0);
            out_sets[base + lane] = st[lane];
            __syncwarp();
            if (lane < cnt - 32) st[lane] = st[32 + lane];
            cnt -= 32;
            __syncwarp();
        }
        if (has && r + 1 < r1) s = gosper_next(s);
    }
    if (cnt > 0) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&lc->n_sets, cnt);
        base = __shfl_sync(kFull, base, 0);
        if (lane < cnt) out_sets[base + lane] = st[lane];
    }
}

// ---------------------------------------------------------------------------
// k_level_sets: the connected k-sets, by whichever enumeration is cheaper for
// this level (decided on the device from the previous level's count):
//   * extension: every connected (k-1)-set plus each of its neighbours; a
//     test-and-set bitmap over all 2^n sets keeps the first producer of each
//     k-set (work ~ count(k-1) * |neighbours|, for sparse graphs far below
//     C(n,k));
//   * filter: combinadic unrank + Gosper stepping over all C(n,k) subsets with
//     the connectivity test (as k_filter; dense graphs).
// Both produce the same set of connected k-sets; their order in the level list
// does not affect the result (each set's best join is computed independently).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_level_sets(const uint32_t *__restrict__ blob,
                                                       const uint32_t *__restrict__ binom_g, int n, int k,
                                                       unsigned long long total, uint32_t per_thread,
                                                       const uint32_t *__restrict__ prev_sets,
                                                       const LevelCounters *__restrict__ prev_lc,
                                                       uint32_t *__restrict__ bitmap, uint32_t *__restrict__ out_sets,
                                                       LevelCounters *__restrict__ lc) {
    __shared__ uint32_t adj[kMaxRels];
    __shared__ uint32_t binom[33 * 33];
    __shared__ uint32_t stage[kWarpsPerBlock][64];
    const uint32_t c_prev = (k == 2) ? (uint32_t)n : __ldcg(&prev_lc->n_sets);
    // per candidate the extension costs a neighbourhood scan share plus one
    // L2 atomic; the filter a Gosper step plus a short connectivity test
    const bool use_ext = (uint64_t)c_prev * (uint64_t)(k + 4 * (n - k + 1)) < total * 3ull;
    // the grid is sized for the filter; the extension needs one thread per
    // set of the previous level, so surplus blocks leave at once
    if (use_ext && (uint64_t)blockIdx.x * blockDim.x >= (uint64_t)c_prev) return;
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob);
    for (int i = threadIdx.x; i < kMaxRels; i += blockDim.x) adj[i] = (i < n) ? h->adj[i] : 0u;
    if (!use_ext)
        for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) binom[i] = binom_g[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *st = stage[warp];
    uint32_t cnt = 0;
    auto emit = [&](bool ok, uint32_t s) {
        uint32_t m = __ballot_sync(kFull, ok);
        if (ok) st[cnt + __popc(m & ((1u << lane) - 1u))] = s;
        cnt += __popc(m);
        __syncwarp();
        if (cnt >= 32) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&lc->n_sets, 32u);
            base = __shfl_sync(kFull, base, 0);
            out_sets[base + lane] = st[lane];
            __syncwarp();
            if (lane < cnt - 32) st[lane] = st[32 + lane];
            cnt -= 32;
            __syncwarp();
        }
    };
    if (use_ext) {
        const uint32_t used_blocks = (uint32_t)min((uint64_t)gridDim.x, ((uint64_t)c_prev + blockDim.x - 1) / blockDim.x);
        const uint32_t nthreads = used_blocks * blockDim.x;
        const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
        // warp-uniform trip count over the previous level
        const uint32_t rounds = (c_prev + nthreads - 1u) / nthreads;
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t idx = tid + r * nthreads;
            uint32_t S = 0u, N = 0u;
            if (idx < c_prev) {
                S = (k == 2) ? (1u << idx) : __ldcg(prev_sets + idx);
                uint32_t x = S;
                while (x) {
                    int v = __ffs(x) - 1;
                    x &= x - 1u;
                    N |= adj[v];
                }
                N &= ~S;
            }
            const int deg = __popc(N);
            const int maxdeg = (int)__reduce_max_sync(kFull, (uint32_t)deg);
            for (int j = 0; j < maxdeg; j++) {
                bool ok = false;
                uint32_t T = 0u;
                if (j < deg) {
                    const uint32_t bitv = N & (0u - N);
                    N ^= bitv;
                    T = S | bitv;
                    const uint32_t bm = 1u << (T & 31u);
                    ok = !(atomicOr(&bitmap[T >> 5], bm) & bm);
                }
                emit(ok, T);
            }
        }
    } else {
        uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        uint64_t r0 = tid * per_thread;
        uint64_t r1 = r0 + per_thread < total ? r0 + per_thread : total;
        uint32_t s = r0 < total ? unrank_ksubset(r0, n, k, binom) : 0u;
        for (uint32_t j = 0; j < per_thread; j++) {
            uint64_t r = r0 + j;
            bool has = r < r1;
            bool ok = has && is_connected(s, adj);
            emit(ok, s);
            if (has && r + 1 < r1) s = gosper_next(s);
        }
    }
    if (cnt > 0) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&lc->n_sets, cnt);
        base = __shfl_sync(kFull, base, 0);
        if (lane < cnt) out_sets[base + lane] = st[lane];
    }
}

// ---------------------------------------------------------------------------
// candidate enumeration + evaluation shared by k_eval / k_ovf_chunks
// ---------------------------------------------------------------------------
struct LaneBest {
    unsigned long long key;
    RelVal val;
    uint32_t left;
    uint32_t first_p;
    bool first_nan;
    RelVal nan_val;
    uint32_t nan_left;
    uint32_t n_valid;

    __device__ __forceinline__ void init() {
        key = ~0ull;
        left = 0;
        first_p = kFull;
        first_nan = false;
        nan_left = 0;
        n_valid = 0;
    }
};

// one valid candidate p = (outer L, inner side) with its cost: the lane keeps
// its first strict minimum (key (ordered cost, p)) and its first candidate
// in enumeration order with that candidate's NaN status
__device__ __forceinline__ void best_update(LaneBest &best, uint32_t p, uint32_t L, const RelVal &out) {
    const bool nan = isnan(out.total);
    best.n_valid++;
    if (p < best.first_p) {
        best.first_p = p;
        best.first_nan = nan;
        if (nan) {
            best.nan_val = out;
            best.nan_left = L;
        }
    }
    if (!nan) {
        const unsigned long long key = ((unsigned long long)ord_float(out.total) << 32) | p;
        if (key < best.key) {
            best.key = key;
            best.val = out;
            best.left = L;
        }
    }
}

__device__ __forceinline__ void evaluate_pair(const DevInfoView &d, const float4 *memo, uint32_t p, uint32_t L,
                                              uint32_t R, LaneBest &b) {
    const RelVal l = load_rel(memo, L, d.h->hz_packed);
    const RelVal r = load_rel(memo, R, d.h->hz_packed);
    best_update(b, p, L, join_eval(d, L, l, R, r));
}

// A valid split (L, R) of a plain-DPsub set and its mirror (R, L), costed in
// one pass (join_eval_mirror); p and pm are their indices in the reference's
// enumeration order.
__device__ __forceinline__ void evaluate_mirror(const DevInfoView &d, const float4 *memo, uint32_t p, uint32_t pm,
                                                uint32_t L, uint32_t R, LaneBest &b) {
    const RelVal l = load_rel(memo, L, d.h->hz_packed);
    const RelVal r = load_rel(memo, R, d.h->hz_packed);
    RelVal out_lr, out_rl;
    join_eval_mirror(d, L, l, R, r, out_lr, out_rl);
    best_update(b, p, L, out_lr);
    best_update(b, pm, R, out_rl);
}

// Plain DPsub over mirror pairs: the reference visits L = pdep(p + 1, S) for
// p = 0 .. P - 1 (P = 2^|S| - 2, gpuqo_cpu_dpsub.cu:32-78), and candidate
// P - 1 - p is the complement of candidate p.  Lanes take contiguous slices
// of [lo, hi) within [0, P / 2); each h names the split L = pdep(h + 1, S)
// and its mirror, both connected or neither, costed together and keyed by
// their own indices h and P - 1 - h.  With ccc the valid splits go through
// the per-warp queue and are costed 32 at a time (the reference's CCC,
// gpuqo_dpsub.cuh:193-259, as a compaction queue).
__device__ __forceinline__ void eval_range_dpsub(const DevInfoView &d, const uint32_t *adj, uint32_t S, uint32_t P,
                                                 uint32_t lo, uint32_t hi, const float4 *memo, uint32_t *q,
                                                 bool ccc, LaneBest &best) {
    const int lane = threadIdx.x & 31;
    const uint32_t span = hi - lo;
    const uint32_t per = (span + 31u) / 32u;
    uint32_t my_lo = lo + per * lane;
    if (my_lo > hi) my_lo = hi;
    const uint32_t my_hi = my_lo + per < hi ? my_lo + per : hi;
    uint32_t h = my_lo;
    uint32_t L = h < my_hi ? pdep32(h + 1u, S) : 0u;
    int qn = 0;   // warp-uniform queue length
    while (__any_sync(kFull, h < my_hi)) {
        const bool has = h < my_hi;
        bool valid = false;
        uint32_t cl = 0, cr = 0;
        if (has) {
            cl = L;
            cr = S ^ L;
            valid = is_connected(cl, adj) && is_connected(cr, adj);
            L = next_subset(L, S);
        }
        const uint32_t ch = h;
        if (has) h++;
        if (!ccc) {
            if (valid) evaluate_mirror(d, memo, ch, P - 1u - ch, cl, cr, best);
            continue;
        }
        const uint32_t m = __ballot_sync(kFull, valid);
        if (valid) {
            const int pos = qn + __popc(m & ((1u << lane) - 1u));
            q[pos * 3 + 0] = ch;
            q[pos * 3 + 1] = cl;
            q[pos * 3 + 2] = cr;
        }
        qn += __popc(m);
        __syncwarp();
        if (qn >= 32) {
            const int pos = qn - 32 + lane;
            const uint32_t eh = q[pos * 3 + 0], el = q[pos * 3 + 1], er = q[pos * 3 + 2];
            __syncwarp();
            qn -= 32;
            evaluate_mirror(d, memo, eh, P - 1u - eh, el, er, best);
        }
    }
    if (ccc && qn > 0) {
        __syncwarp();
        if (lane < qn) evaluate_mirror(d, memo, q[lane * 3 + 0], P - 1u - q[lane * 3 + 0], q[lane * 3 + 1],
                                       q[lane * 3 + 2], best);
    }
    __syncwarp();
}

// Enumerates candidate indices [lo, hi) of set S (lanes take contiguous
// slices), tests each candidate, and evaluates the valid ones.  With ccc the
// valid candidates go through a per-warp queue and are evaluated 32 at a time
// (the reference's CCC, gpuqo_dpsub.cuh:193-259, as a compaction queue).
template <int MODE>
__device__ __forceinline__ void eval_range(const DevInfoView &d, const uint32_t *adj, uint32_t S, const Blocks &B,
                                           uint32_t lo, uint32_t hi, const float4 *memo, uint32_t *q, bool ccc,
                                           LaneBest &best) {
    const int lane = threadIdx.x & 31;
    uint32_t span = hi - lo;
    uint32_t per = (span + 31u) / 32u;
    uint32_t my_lo = lo + per * lane;
    uint32_t my_hi = my_lo + per < hi ? my_lo + per : hi;
    if (my_lo > hi) my_lo = hi;
    uint32_t p = my_lo;
    // iterator state
    uint32_t L = 0;           // MODE 0: current left subset
    int b = 0;                // MODE 1: block index
    uint32_t lb = 0;          // MODE 1: current subset of block b
    uint32_t key = 0;         // MODE 1: the reference's index of the candidate
    CycleCache cc;            // MODE 1: arcs of the current cycle block
    if (p < my_hi) {
        if (MODE == kModeDpsub) {
            L = pdep32(p + 1u, S);
        } else {
            // p counts enumerated candidates (Blocks::eprefix); cycle blocks
            // decode their arcs per candidate, other blocks walk nextSubset
            while (b + 1 < B.nb && B.eprefix[b + 1] <= p) b++;
            if (!((B.cyc >> b) & 1u)) lb = pdep32(p - B.eprefix[b] + 1u, B.mask[b]);
        }
    }
    int qn = 0;   // warp-uniform queue length
    while (__any_sync(kFull, p < my_hi)) {
        bool has = p < my_hi;
        bool valid = false;
        uint32_t cl = 0, cr = 0;
        if (has) {
            if (MODE == kModeDpsub) {
                cl = L;
                cr = S ^ L;
                valid = is_connected(cl, adj) && is_connected(cr, adj);
                L = next_subset(L, S);
            } else {
                const uint32_t blk = B.mask[b];
                const bool cyc = (B.cyc >> b) & 1u;
                if (cyc) lb = cached_arc(cc, S, b, blk, adj, p - B.eprefix[b]);
                uint32_t rb = blk ^ lb;
                if (cyc && blk == S) {   // the set is the cycle: arc and complement
                    cl = lb;
                    cr = rb;
                } else {
                    cl = grow(lowest(lb), S & ~rb, adj);
                    cr = grow(lowest(rb), S & ~lb, adj);
                }
                valid = (cl | cr) == S;
                // the reference's index of this candidate (Blocks::prefix space)
                key = B.prefix[b] + (cyc ? pext32(lb, blk) - 1u : p - B.eprefix[b]);
                if (p + 1u < B.eprefix[b + 1]) {
                    if (!cyc) lb = next_subset(lb, blk);
                } else if (b + 1 < B.nb) {
                    b++;
                    lb = lowest(B.mask[b]);
                }
            }
        }
        uint32_t cp = (MODE == kModeMpdp) ? key : p;
        if (MODE == kModeMpdp && valid) cp = key_index(*d.h, key, cl, S);
        if (has) p++;
        if (!ccc) {
            if (valid) evaluate_pair(d, memo, cp, cl, cr, best);
            continue;
        }
        uint32_t m = __ballot_sync(kFull, valid);
        if (valid) {
            int pos = qn + __popc(m & ((1u << lane) - 1u));
            q[pos * 3 + 0] = cp;
            q[pos * 3 + 1] = cl;
            q[pos * 3 + 2] = cr;
        }
        qn += __popc(m);
        __syncwarp();
        if (qn >= 32) {
            int pos = qn - 32 + lane;
            uint32_t ep = q[pos * 3 + 0], el = q[pos * 3 + 1], er = q[pos * 3 + 2];
            __syncwarp();
            qn -= 32;
            evaluate_pair(d, memo, ep, el, er, best);
        }
    }
    if (ccc && qn > 0) {
        __syncwarp();
        if (lane < qn) evaluate_pair(d, memo, q[lane * 3 + 0], q[lane * 3 + 1], q[lane * 3 + 2], best);
    }
    __syncwarp();
}

struct WarpWinner {
    bool is_writer;
    bool use_nan;
};

__device__ __forceinline__ WarpWinner warp_winner(const LaneBest &b, unsigned long long &min_key,
                                                  unsigned long long &first_key) {
    uint32_t kh = (uint32_t)(b.key >> 32), kl = (uint32_t)b.key;
    uint32_t mh = __reduce_min_sync(kFull, kh);
    uint32_t ml = __reduce_min_sync(kFull, kh == mh ? kl : kFull);
    uint32_t mf = __reduce_min_sync(kFull, b.first_p);
    bool nan_first = (b.first_p == mf) && b.first_nan;
    unsigned nm = __ballot_sync(kFull, nan_first);
    min_key = ((unsigned long long)mh << 32) | ml;
    first_key = ((unsigned long long)mf << 1) | (nm ? 1ull : 0ull);
    WarpWinner w;
    if (nm) {
        w.is_writer = nan_first;
        w.use_nan = true;
    } else {
        w.is_writer = (b.key == min_key) && (b.key != ~0ull);
        w.use_nan = false;
    }
    return w;
}

__device__ __forceinline__ void memo_write(const DevHeader &h, float4 *memo, uint32_t *memo_left, uint32_t S,
                                           const RelVal &v, uint32_t left) {
    memo[S] = make_float4(v.rows, v.startup, v.total, __uint_as_float(memo_width_word(h, v.rows, v.width)));
    memo_left[S] = left;
}

__device__ __forceinline__ void load_blob_to_smem(const uint32_t *blob, uint32_t words, uint32_t *sm) {
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) sm[i] = blob[i];
    __syncthreads();
}

// ---------------------------------------------------------------------------
// k_eval: one warp per connected set
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_eval(const uint32_t *__restrict__ blob, uint32_t blob_words, int k,
                                                 const uint32_t *__restrict__ sets, LevelCounters *__restrict__ lc,
                                                 float4 *__restrict__ memo, uint32_t *__restrict__ memo_left,
                                                 uint32_t *__restrict__ ovf_set, uint32_t *__restrict__ ovf_P,
                                                 uint32_t *__restrict__ ovf_off,
                                                 unsigned long long *__restrict__ ovf_key,
                                                 unsigned long long *__restrict__ ovf_first,
                                                 GlobalCounters *__restrict__ glob, int ccc,
                                                 const uint32_t *__restrict__ count_ptr = nullptr) {
    const uint32_t count = count_ptr ? *count_ptr : lc->n_sets;
    if (count == 0u) return;
    extern __shared__ __align__(16) uint32_t sm[];
    load_blob_to_smem(blob, blob_words, sm);
    const DevInfoView d = make_view(sm);
    const uint32_t *adj = d.h->adj;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *q = sm + ((blob_words + 3u) & ~3u) + warp * kQueueWords;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    unsigned long long pairs = 0;
    Blocks B;
    B.nb = 0;
    for (uint32_t i = blockIdx.x * kWarpsPerBlock + warp; i < count; i += nwarps) {
        const uint32_t S = sets[i];
        uint32_t P;
        if (MODE == kModeDpsub) {
            P = (1u << k) - 2u;
        } else {
            find_blocks(S, adj, B);
            P = B.etotal;
        }
        if (P > kOvfLimit) {
            if (lane == 0) {
                uint32_t nch = (ovf_work(MODE, P) + kChunk - 1u) / kChunk;
                unsigned long long old = atomicAdd(&lc->ovf_packed, (1ull << 40) | (unsigned long long)nch);
                uint32_t idx = (uint32_t)(old >> 40);
                ovf_set[idx] = S;
                ovf_P[idx] = P;
                ovf_off[idx] = (uint32_t)(old & 0xFFFFFFFFFFull);
                ovf_key[idx] = ~0ull;
                ovf_first[idx] = ~0ull;
            }
            continue;
        }
        LaneBest best;
        best.init();
        if constexpr (MODE == kModeDpsub) eval_range_dpsub(d, adj, S, P, 0u, P / 2u, memo, q, ccc != 0, best);
        else eval_range<MODE>(d, adj, S, B, 0u, P, memo, q, ccc != 0, best);
        unsigned long long mk, fk;
        WarpWinner w = warp_winner(best, mk, fk);
        if (w.is_writer) {
            if (w.use_nan) memo_write(*d.h, memo, memo_left, S, best.nan_val, best.nan_left);
            else memo_write(*d.h, memo, memo_left, S, best.val, best.left);
        }
        pairs += best.n_valid;
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

// ---------------------------------------------------------------------------
// k_eval_mpdp: MPDP with G lanes per connected set (32/G sets per warp).
// G is picked on the device from the level's set count so that small levels
// still fill the GPU and large levels do not pay the per-set block search 32
// times per warp.  Lanes of a group take candidates p = g, g+G, ...; the loop
// runs the warp's maximum trip count so the group reductions can use
// full-warp shuffles.
// ---------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ void mpdp_groups(const DevInfoView &d, const uint32_t *adj, uint32_t first_set,
                                            uint32_t stride_sets, const uint32_t *sets, uint32_t count,
                                            LevelCounters *lc, float4 *memo, uint32_t *memo_left,
                                            uint32_t *ovf_set, uint32_t *ovf_P, uint32_t *ovf_off,
                                            unsigned long long *ovf_key, unsigned long long *ovf_first,
                                            unsigned long long &pairs) {
    const int lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const uint32_t group_mask = (G == 32) ? kFull : (((1u << G) - 1u) << (grp * G));
    Blocks B;
    CycleCache cc;
    for (uint32_t base = first_set; base < count; base += stride_sets) {
        const uint32_t i = base + (uint32_t)grp;
        const bool has = i < count;
        const uint32_t S = has ? sets[i] : 0u;
        uint32_t P = 0;
        B.nb = 0;
        if (has) {
            find_blocks(S, adj, B);
            P = B.etotal;
        }
        __syncwarp();
        const bool ovf = has && P > kOvfLimit;
        if (ovf && gl == 0) {
            uint32_t nch = (P + kChunk - 1u) / kChunk;
            unsigned long long old = atomicAdd(&lc->ovf_packed, (1ull << 40) | (unsigned long long)nch);
            uint32_t idx = (uint32_t)(old >> 40);
            ovf_set[idx] = S;
            ovf_P[idx] = P;
            ovf_off[idx] = (uint32_t)(old & 0xFFFFFFFFFFull);
            ovf_key[idx] = ~0ull;
            ovf_first[idx] = ~0ull;
        }
        const uint32_t myP = (has && !ovf) ? P : 0u;
        const uint32_t iters = __reduce_max_sync(kFull, (myP + G - 1u) / G);
        LaneBest best;
        best.init();
        int b = 0;
        for (uint32_t it = 0; it < iters; it++) {
            const uint32_t p = (uint32_t)gl + it * G;
            if (p < myP) {
                uint32_t L, R;
                uint32_t key;
                if (mpdp_candidate(S, B, adj, p, b, L, R, key, cc))
                    evaluate_pair(d, memo, key_index(*d.h, key, L, S), L, R, best);
            }
        }
        // group reduction: min key, min first candidate (NaN rule)
        uint32_t kh = (uint32_t)(best.key >> 32), kl = (uint32_t)best.key, fp = best.first_p;
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) {
            uint32_t oh = __shfl_xor_sync(kFull, kh, off);
            uint32_t ol = __shfl_xor_sync(kFull, kl, off);
            uint32_t of = __shfl_xor_sync(kFull, fp, off);
            if (oh < kh || (oh == kh && ol < kl)) {
                kh = oh;
                kl = ol;
            }
            if (of < fp) fp = of;
        }
        const bool nan_first = has && !ovf && best.first_p == fp && best.first_nan;
        const unsigned nm = __ballot_sync(kFull, nan_first) & group_mask;
        const unsigned long long gkey = ((unsigned long long)kh << 32) | kl;
        if (has && !ovf) {
            if (nm) {
                if (nan_first) memo_write(*d.h, memo, memo_left, S, best.nan_val, best.nan_left);
            } else if (best.key == gkey && best.key != ~0ull) {
                memo_write(*d.h, memo, memo_left, S, best.val, best.left);
            }
        }
        pairs += best.n_valid;
    }
}

__global__ void __launch_bounds__(kBlock) k_eval_mpdp(const uint32_t *__restrict__ blob, uint32_t blob_words,
                                                      const uint32_t *__restrict__ sets,
                                                      LevelCounters *__restrict__ lc, float4 *__restrict__ memo,
                                                      uint32_t *__restrict__ memo_left, uint32_t *__restrict__ ovf_set,
                                                      uint32_t *__restrict__ ovf_P, uint32_t *__restrict__ ovf_off,
                                                      unsigned long long *__restrict__ ovf_key,
                                                      unsigned long long *__restrict__ ovf_first,
                                                      GlobalCounters *__restrict__ glob, uint32_t target_lanes,
                                                      int max_group) {
    extern __shared__ __align__(16) uint32_t sm[];
    load_blob_to_smem(blob, blob_words, sm);
    const DevInfoView d = make_view(sm);
    const uint32_t *adj = d.h->adj;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t count = lc->n_sets;
    // lanes per set: enough lanes in flight to fill the GPU, no more than the
    // largest useful group for this level
    int G = 1;
    while (G < max_group && (uint64_t)count * (uint64_t)G < (uint64_t)target_lanes) G <<= 1;
    const uint32_t gwarp = blockIdx.x * kWarpsPerBlock + warp;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    unsigned long long pairs = 0;
    switch (G) {
#define GQB_G(g)                                                                                                  \
    case g:                                                                                                       \
        mpdp_groups<g>(d, adj, gwarp * (32 / g), nwarps * (32 / g), sets, count, lc, memo, memo_left, ovf_set,   \
                       ovf_P, ovf_off, ovf_key, ovf_first, pairs);                                                \
        break;
        GQB_G(1)
        GQB_G(2)
        GQB_G(4)
        GQB_G(8)
        GQB_G(16)
        GQB_G(32)
#undef GQB_G
    default:
        break;
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

// ---------------------------------------------------------------------------
// k_eval_tree: MPDP on a tree-shaped query graph (star, snowflake, chain, and
// the contracted trees of IDP sub-problems), any relation numbering.
// A connected set S is a subtree; the reference's block search walks it from
// its lowest relation r, and every block is a bridge {a, b}, a < b.  With the
// query tree rooted at r, let c be the child end of the edge: removing the
// edge leaves S & sub_r[c] and the rest, so no DFS is needed.  Candidate
// order: blocks are emitted in post-order of their child end, and the
// reference's enumeration index is 2 * post_r(c) + (lb == {a} ? 0 : 1) with
//     post_r(c) = |S & before_r[c]| - |S & anc_r[c]| + |S & sub_r[c]| - 1
// (preorder rank minus depth plus subtree size minus one).  With ec_masked
// only the classes on edge {a, b} can match.
// ---------------------------------------------------------------------------
struct EdgeIter {
    uint32_t vs;      // vertices of S not yet started
    uint32_t nb;      // remaining higher neighbours of v
    int v;
    uint32_t e;       // index of the next edge to be returned
};

__device__ __forceinline__ void edge_next(const uint32_t *adj, uint32_t S, EdgeIter &it, int &a, int &b) {
    while (it.nb == 0u) {
        it.v = __ffs(it.vs) - 1;
        it.vs &= it.vs - 1u;
        it.nb = adj[it.v] & S & ~((2u << it.v) - 1u);
    }
    a = it.v;
    b = __ffs(it.nb) - 1;
    it.nb &= it.nb - 1u;
    it.e++;
}

// Edge-wise evaluation: the candidates of S come in mirror pairs, c = 2e and
// c = 2e + 1 being the two orientations of split edge e (side 0 puts the
// component of a on the outer side).  A lane takes whole edges: it decodes
// the edge once, loads the two memo entries once and costs both orientations
// in one fused pass (join_eval_mirror_tree: shared class visit, two
// independent cost chains), keyed by the reference's indices of both
// candidates.  Lanes of a group take edges e = gl, gl + G, ...
// PIPE: software-pipelined edge loop for G < 32, in the 2- and 3-blocks
// persistent kernels (the next edge's memo entries are requested before the
// current edge is costed); at 64 registers (the 4-blocks persistent kernel and
// the per-level kernel) it spills, and those keep the plain loop.
template <int G, bool MASKED, bool PIPE>
__device__ __forceinline__ void tree_groups(const DevInfoView &d, uint32_t first_set, uint32_t stride_sets,
                                            const uint32_t *sets, uint32_t count, int k, float4 *memo,
                                            uint32_t *memo_left, unsigned long long &pairs) {
    const DevHeader &h = *d.h;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const uint32_t group_mask = (G == 32) ? kFull : (((1u << G) - 1u) << (grp * G));
    const uint32_t E = (uint32_t)(k - 1);                 // split edges of a k-set
    const uint32_t per_lane = (E + G - 1u) / G;
    // plain-DPsub index of the mirror: pext(S - L, S) - 1 = 2^k - 3 - p
    const uint32_t mirror_base = (k >= 32 ? 0xFFFFFFFFu : ((1u << k) - 1u)) - 2u;
    for (uint32_t base = first_set; base < count; base += stride_sets) {
        const uint32_t i = base + (uint32_t)grp;
        const bool has = i < count;
        const uint32_t S = has ? __ldcg(sets + i) : 0u;
        EdgeIter it;
        it.vs = S;
        it.nb = 0u;
        it.v = 0;
        it.e = 0u;
        int a = 0, b = 0;
        // G == 32 (one set per warp): the edges of S indexed cooperatively.
        // Lane t takes the t-th relation of S and its higher-numbered
        // neighbours in S; the inclusive prefix of their counts numbers the
        // edges in edge_next's order (lower end, then higher end), so an
        // edge is found by a binary search over the lanes instead of walking
        // the edges before it.
        int vt = 0;
        uint32_t fwd = 0u, scan = 0u;
        if (G == 32) {
            const int kk = __popc(S);
            if (lane < kk) {
                vt = (int)__fns(S, 0u, lane + 1);
                fwd = h.adj[vt] & S & ~((2u << vt) - 1u);
            }
            scan = (uint32_t)__popc(fwd);
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t o = __shfl_up_sync(kFull, scan, off);
                if (lane >= off) scan += o;
            }
        }
        LaneBest best;
        best.init();
        const uint32_t *tab = reinterpret_cast<const uint32_t *>(d.h) + h.tree_tab;
        const int n = h.n, nn = n * n;
        // split edge (a, b): the side holding a (outer in orientation 0), the
        // reference's indices of both orientations and the classes on the edge
        auto decode = [&](uint32_t &L0, uint32_t &p0, uint32_t &p1, uint32_t &ecm) {
            const int rt = __ffs(S) - 1;
            const uint32_t *anc_r = tab + 2 * nn + rt * n;
            const int ch = ((anc_r[b] >> a) & 1u) ? b : a;        // child end w.r.t. root rt
            const uint32_t comp_c = S & tab[rt * n + ch];
            L0 = (ch == a) ? comp_c : (S ^ comp_c);
            const uint32_t post = (uint32_t)(__popc(S & tab[nn + rt * n + ch]) - __popc(S & anc_r[ch]) +
                                             __popc(comp_c) - 1);
            if (h.index_order) {
                p0 = dpsub_index(L0, S);
                p1 = mirror_base - p0;
            } else {
                p0 = 2u * post;
                p1 = p0 + 1u;
            }
            ecm = 0u;
            if (MASKED) {
                const int ch0 = ((tab[2 * nn + b] >> a) & 1u) ? b : a;   // child end w.r.t. relation 0
                ecm = h.edge_ec[ch0];
            }
        };
        // costs both orientations of one edge from its two memo entries
        auto cost2 = [&](uint32_t L0, uint32_t p0, uint32_t p1, uint32_t ecm, const float4 lv, const float4 rv) {
            const uint32_t R0 = S ^ L0;
            const RelVal l = unpack_rel(lv, h.hz_packed), r = unpack_rel(rv, h.hz_packed);
            RelVal o0, o1;
            join_eval_mirror_tree<MASKED>(d, L0, l, R0, r, ecm, o0, o1);
            best_update(best, p0, L0, o0);
            best_update(best, p1, R0, o1);
        };
        if (G != 32 && !PIPE) {
            for (uint32_t j = 0; j < per_lane; j++) {
                const uint32_t e = (uint32_t)gl + j * G;
                if (has && e < E) {
                    while (it.e <= e) edge_next(h.adj, S, it, a, b);
                    uint32_t L0, p0, p1, ecm;
                    decode(L0, p0, p1, ecm);
                    cost2(L0, p0, p1, ecm, __ldcg(memo + L0), __ldcg(memo + (S ^ L0)));
                }
            }
        } else if (G != 32) {
            uint32_t cL = 0u, cp0 = 0u, cp1 = 0u, cecm = 0u;
            float4 clv = make_float4(0.f, 0.f, 0.f, 0.f), crv = clv;
            bool cact = false;
            auto fetch = [&](uint32_t j, uint32_t &L0, uint32_t &p0, uint32_t &p1, uint32_t &ecm, float4 &lv,
                             float4 &rv) -> bool {
                const uint32_t e = (uint32_t)gl + j * G;
                if (!(has && e < E)) return false;
                while (it.e <= e) edge_next(h.adj, S, it, a, b);
                decode(L0, p0, p1, ecm);
                lv = __ldcg(memo + L0);
                rv = __ldcg(memo + (S ^ L0));
                return true;
            };
            if (per_lane > 0) cact = fetch(0u, cL, cp0, cp1, cecm, clv, crv);
            for (uint32_t j = 0; j < per_lane; j++) {
                uint32_t nL = 0u, np0 = 0u, np1 = 0u, necm = 0u;
                float4 nlv = clv, nrv = crv;
                const bool nact = (j + 1 < per_lane) ? fetch(j + 1, nL, np0, np1, necm, nlv, nrv) : false;
                if (cact) cost2(cL, cp0, cp1, cecm, clv, crv);
                cL = nL;
                cp0 = np0;
                cp1 = np1;
                cecm = necm;
                clv = nlv;
                crv = nrv;
                cact = nact;
            }
        } else {
            for (uint32_t j = 0; j < per_lane; j++) {
                const uint32_t e = (uint32_t)gl + j * G;
                const bool active = has && e < E;
                // smallest lane t with scan_t > e (every lane takes part in the shuffles)
                int lo = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const uint32_t sv = __shfl_sync(kFull, scan, lo + step - 1);
                    if (sv <= e) lo += step;
                }
                const int t = lo > 31 ? 31 : lo;
                const uint32_t before = __shfl_sync(kFull, scan, t) - (uint32_t)__popc(__shfl_sync(kFull, fwd, t));
                const uint32_t ft = __shfl_sync(kFull, fwd, t);
                a = __shfl_sync(kFull, vt, t);
                if (active) {
                    b = (int)__fns(ft, 0u, (int)(e - before) + 1);
                    uint32_t L0, p0, p1, ecm;
                    decode(L0, p0, p1, ecm);
                    cost2(L0, p0, p1, ecm, __ldcg(memo + L0), __ldcg(memo + (S ^ L0)));
                }
            }
        }
        uint32_t kh = (uint32_t)(best.key >> 32), kl = (uint32_t)best.key, fp = best.first_p;
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) {
            uint32_t oh = __shfl_xor_sync(kFull, kh, off);
            uint32_t ol = __shfl_xor_sync(kFull, kl, off);
            uint32_t of = __shfl_xor_sync(kFull, fp, off);
            if (oh < kh || (oh == kh && ol < kl)) {
                kh = oh;
                kl = ol;
            }
            if (of < fp) fp = of;
        }
        const bool nan_first = has && best.first_p == fp && best.first_nan;
        const unsigned nm = __ballot_sync(kFull, nan_first) & group_mask;
        const unsigned long long gkey = ((unsigned long long)kh << 32) | kl;
        if (has) {
            if (nm) {
                if (nan_first) memo_write(*d.h, memo, memo_left, S, best.nan_val, best.nan_left);
            } else if (best.key == gkey && best.key != ~0ull) {
                memo_write(*d.h, memo, memo_left, S, best.val, best.left);
            }
        }
        pairs += best.n_valid;
    }
}

__global__ void __launch_bounds__(kBlock, 4) k_eval_tree(const uint32_t *__restrict__ blob, uint32_t blob_words, int k,
                                                      const uint32_t *__restrict__ sets,
                                                      LevelCounters *__restrict__ lc, float4 *__restrict__ memo,
                                                      uint32_t *__restrict__ memo_left,
                                                      GlobalCounters *__restrict__ glob, uint32_t target_lanes,
                                                      int max_group) {
    extern __shared__ __align__(16) uint32_t sm[];
    load_blob_to_smem(blob, blob_words, sm);
    const DevInfoView d = make_view(sm);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t count = lc->n_sets;
    // group sizes 2, 8 or 32 (fewer instantiations keep the code in the
    // instruction cache)
    int G = 2;
    while (G < max_group && (uint64_t)count * (uint64_t)G < (uint64_t)target_lanes) G <<= 1;
    G = G <= 2 ? 2 : (G <= 8 ? 8 : 32);
    const uint32_t gwarp = blockIdx.x * kWarpsPerBlock + warp;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    const bool masked = d.h->ec_masked != 0u;
    unsigned long long pairs = 0;
    switch (G * 2 + (masked ? 1 : 0)) {
#define GQB_T(g)                                                                                                 \
    case 2 * g:                                                                                                  \
        tree_groups<g, false, false>(d, gwarp * (32 / g), nwarps * (32 / g), sets, count, k, memo,               \
                                     memo_left, pairs);                                                          \
        break;                                                                                                   \
    case 2 * g + 1:                                                                                              \
        tree_groups<g, true, false>(d, gwarp * (32 / g), nwarps * (32 / g), sets, count, k, memo,                \
                                     memo_left, pairs);                                                          \
        break;
        GQB_T(2)
        GQB_T(8)
        GQB_T(32)
#undef GQB_T
    default:
        break;
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

// ---------------------------------------------------------------------------
// k_dp_tree: the whole MPDP of a tree-shaped query in ONE cooperative,
// persistent launch.  The planner info and the binomial table are staged in
// shared memory once; levels are separated by a grid barrier, and each phase
// evaluates level k while enumerating level k+1 (independent: the
// enumeration reads only level k's sets).  Data written by other blocks is
// read with ld.global.cg (L2), never through a possibly stale L1 line.
// The barrier spins a bounded number of times; on timeout it raises an error
// flag, every block leaves, and the host reruns the DP with per-level
// launches.
// ---------------------------------------------------------------------------
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;   // 4 s of global time
constexpr unsigned kBarrierSpinLimit = 1u << 26;                  // hard cap on polls as well (~30 s)

// poll limit of one barrier wait: the launch argument when non-zero (the
// gpuqo_b200_barrier_poll_limit setting, which makes waits run out on purpose
// so that the timeout path can be exercised), else kBarrierSpinLimit
__device__ __forceinline__ unsigned barrier_polls(unsigned poll_limit) {
    return poll_limit != 0u ? poll_limit : kBarrierSpinLimit;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bar[0] = arrivals, bar[2] = error flag (both zero at launch).  The arrival
// counter only grows: a block's e-th barrier of the launch completes when it
// reaches e * gridDim.x, so nobody resets it and the last block to arrive has
// nothing more to do.  Thread 0 arrives with a gpu-scope release reduction
// (ordering every write its block made before the __syncthreads) and polls
// with gpu-scope acquire loads (ACQUIRE_POLL), or with relaxed loads and one
// fence once the count is reached: an acquire load also drops the SM's L1
// contents, which a kernel that keeps its working data in shared memory does
// not mind (k_dp_tree: the faster barrier) but which costs the batch kernel,
// whose per-query data is read through L1 while waiting blocks poll on the
// same SM.  The verdict is the same for every thread of the block (thread 0
// decides); blocks may disagree only after a timeout, and then every later
// barrier sees the error flag and returns false at once, so all blocks leave.
// epoch: the caller's count of barriers passed (thread 0); max_polls: polls
// before the wait gives up (barrier_polls).
template <bool ACQUIRE_POLL>
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned &epoch, unsigned max_polls) {
    __shared__ unsigned s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        epoch++;
        const unsigned target = epoch * gridDim.x;
        volatile unsigned *verr = bar + 2;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        const unsigned long long t0 = global_ns();
        unsigned spins = 0;
        for (;;) {
            unsigned c;
            if (ACQUIRE_POLL) {
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(bar) : "memory");
            } else {
                asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(bar) : "memory");
            }
            if (c >= target || *verr != 0u) {
                if (!ACQUIRE_POLL) __threadfence();
                break;
            }
            if (++spins >= max_polls || global_ns() - t0 > kBarrierTimeoutNs) {
                atomicExch(bar + 2, 1u);
                break;
            }
        }
        s_ok = (*verr == 0u) ? 1u : 0u;
    }
    __syncthreads();
    return s_ok != 0u;
}

// One enumeration phase (level k) of a tree-shaped query graph with the
// block's shared adjacency, binomial table and per-warp staging area.
//
// Extension without a dedup structure: adding a neighbour v to a connected
// set S of a tree makes v a leaf of T = S + v (v has exactly one neighbour p
// in S), and every connected T of two or more relations has one largest
// leaf.  T is emitted only from the S whose added v is that largest leaf: the
// other leaves of T are the leaves of S except p (p gains the neighbour v),
// or S itself when S is a single relation.  So each connected k-set appears
// exactly once, with no atomics and no bitmap to clear.
__device__ __forceinline__ void level_sets_phase(const uint32_t *adj, const uint32_t *binom, uint32_t *st, int n,
                                                 int k, const uint32_t *prev_sets, uint32_t c_prev,
                                                 uint32_t *out_sets, LevelCounters *lc) {
    const int lane = threadIdx.x & 31;
    const uint64_t total = binom[n * 33 + k];
    const uint32_t nthreads = gridDim.x * blockDim.x;
    // from the far end of the grid: the first warps evaluate the first sets
    // of the level in the same phase, so small levels split the two jobs
    const uint32_t tid = nthreads - 1u - (blockIdx.x * blockDim.x + threadIdx.x);
    uint32_t cnt = 0;
    auto emit = [&](bool ok, uint32_t s) {
        uint32_t m = __ballot_sync(kFull, ok);
        if (ok) st[cnt + __popc(m & ((1u << lane) - 1u))] = s;
        cnt += __popc(m);
        __syncwarp();
        if (cnt >= 32) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&lc->n_sets, 32u);
            base = __shfl_sync(kFull, base, 0);
            out_sets[base + lane] = st[lane];
            __syncwarp();
            if (lane < cnt - 32) st[lane] = st[32 + lane];
            cnt -= 32;
            __syncwarp();
        }
    };
    const bool use_ext = (uint64_t)c_prev * (uint64_t)(k + 4 * (n - k + 1)) < total * 3ull;
    if (use_ext) {
        const uint32_t rounds = (c_prev + nthreads - 1u) / nthreads;
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t idx = tid + r * nthreads;
            uint32_t S = 0u, N = 0u, leaves = 0u;
            if (idx < c_prev) {
                S = (k == 2) ? (1u << idx) : __ldcg(prev_sets + idx);
                uint32_t x = S;
                while (x) {
                    int v = __ffs(x) - 1;
                    x &= x - 1u;
                    const uint32_t a = adj[v];
                    N |= a;
                    if (__popc(a & S) == 1) leaves |= 1u << v;
                }
                N &= ~S;
            }
            const bool single = (S & (S - 1u)) == 0u;
            const int deg = __popc(N);
            const int maxdeg = (int)__reduce_max_sync(kFull, (uint32_t)deg);
            for (int j = 0; j < maxdeg; j++) {
                bool ok = false;
                uint32_t T = 0u;
                if (j < deg) {
                    const uint32_t bitv = N & (0u - N);
                    N ^= bitv;
                    T = S | bitv;
                    const uint32_t p = adj[__ffs(bitv) - 1] & S;            // v's only neighbour in S
                    const uint32_t others = single ? S : (leaves & ~p);    // the other leaves of T
                    ok = others < bitv;                                     // v is T's largest leaf
                }
                emit(ok, T);
            }
        }
    } else {
        const uint32_t per_thread = (uint32_t)((total + nthreads - 1) / nthreads);
        const uint64_t r0 = (uint64_t)tid * per_thread;
        const uint64_t r1 = r0 + per_thread < total ? r0 + per_thread : total;
        uint32_t s = r0 < total ? unrank_ksubset(r0, n, k, binom) : 0u;
        for (uint32_t j = 0; j < per_thread; j++) {
            const uint64_t r = r0 + j;
            const bool has = r < r1;
            const bool ok = has && is_connected(s, adj);
            emit(ok, s);
            if (has && r + 1 < r1) s = gosper_next(s);
        }
    }
    if (cnt > 0) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&lc->n_sets, cnt);
        base = __shfl_sync(kFull, base, 0);
        if (lane < cnt) out_sets[base + lane] = st[lane];
    }
    __syncwarp();
}

__device__ __forceinline__ void extract_plan(const float4 *memo, const uint32_t *memo_left, uint32_t full,
                                             uint32_t wmask, TreeNode *out, int *n_out) {
    int n = 0;
    uint32_t stack_set[64];
    int stack_parent[64], stack_side[64];
    int sp = 0;
    stack_set[sp] = full;
    stack_parent[sp] = -1;
    stack_side[sp] = 0;
    sp++;
    while (sp > 0 && n < 64) {
        sp--;
        const uint32_t s = stack_set[sp];
        const int parent = stack_parent[sp], side = stack_side[sp];
        const float4 v = __ldcg(memo + s);
        TreeNode t;
        t.set = s;
        t.left = -1;
        t.right = -1;
        t.rows = v.x;
        t.startup = v.y;
        t.total = v.z;
        t.width = (int)(__float_as_uint(v.w) & wmask);
        const int me = n++;
        out[me] = t;
        if (parent >= 0) {
            if (side == 0) out[parent].left = me;
            else out[parent].right = me;
        }
        const uint32_t l = __ldcg(memo_left + s) & s;
        if (__popc(s) > 1 && l != 0u && l != s && sp + 2 <= 64) {
            stack_set[sp] = s ^ l;
            stack_parent[sp] = me;
            stack_side[sp] = 1;
            sp++;
            stack_set[sp] = l;
            stack_parent[sp] = me;
            stack_side[sp] = 0;
            sp++;
        }
    }
    *n_out = n;
}

// MINB: blocks per SM the register budget is set for (2: up to 128
// registers, the cost model without spills and half the barrier arrivals,
// for small and mid-size queries whose levels are latency-bound; 3: 80
// registers; 4: 64 registers, more warps to hide latency on large levels);
// chosen per query from its connected sets per level, the total over the
// relation count (Tuning::single_narrow_level_sets,
// Tuning::single_wide_level_sets)
// MASKED: every class of the query is a two-member class on a tree edge
// (DevHeader::ec_masked), a separate kernel so that each carries only the
// evaluation paths its queries take
template <int MINB, bool MASKED>
__global__ void __launch_bounds__(kBlock, MINB) k_dp_tree(const uint32_t *__restrict__ blob, uint32_t blob_words,
                                                       const uint32_t *__restrict__ binom_g, float4 *__restrict__ memo,
                                                       uint32_t *__restrict__ memo_left, uint32_t *__restrict__ setsA,
                                                       uint32_t *__restrict__ setsB, LevelCounters *__restrict__ lvl,
                                                       GlobalCounters *__restrict__ glob, TreeNode *__restrict__ tree,
                                                       int *__restrict__ tree_n, unsigned *__restrict__ bar,
                                                       uint32_t target_lanes, unsigned poll_limit) {
    extern __shared__ __align__(16) uint32_t sm[];
    const uint32_t bw = (blob_words + 3u) & ~3u;
    const unsigned max_polls = barrier_polls(poll_limit);
    uint32_t *binom = sm + bw;
    uint32_t *stage = binom + 33 * 33 + 3;   // 16-byte aligned (bw, 1092 words)
    for (uint32_t i = threadIdx.x; i < blob_words; i += blockDim.x) sm[i] = blob[i];
    for (uint32_t i = threadIdx.x; i < 33 * 33; i += blockDim.x) binom[i] = binom_g[i];
    __syncthreads();
    const DevInfoView d = make_view(sm);
    const int n = d.h->n;
    const uint32_t *adj = d.h->adj;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *st = stage + warp * 64;
    const uint32_t gwarp = blockIdx.x * kWarpsPerBlock + warp;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    unsigned long long pairs = 0;
    unsigned epoch = 0;   // grid barriers passed (thread 0)
    // the pipelined candidate loop needs the registers of the 2- and 3-blocks
    // variants; at 64 registers it spills and the 4-blocks variant keeps the
    // plain loop
    constexpr bool kPipe = MINB < 4;

    // phase 0: base relations (gpuqo_cpu_sequential.cu:80-92) and level-2 sets
    if (blockIdx.x == 0 && threadIdx.x < n) {
        const int i = threadIdx.x;
        memo[1u << i] = base_entry(*d.h, i);
        memo_left[1u << i] = 0u;
    }
    if (n >= 2) level_sets_phase(adj, binom, st, n, 2, nullptr, (uint32_t)n, setsA, lvl + 2);
    if (!grid_barrier<true>(bar, epoch, max_polls)) return;
    for (int k = 2; k <= n; k++) {
        uint32_t *cur = (k & 1) ? setsB : setsA;
        uint32_t *nxt = (k & 1) ? setsA : setsB;
        const uint32_t count = __ldcg(&lvl[k].n_sets);
        if (k < n) level_sets_phase(adj, binom, st, n, k + 1, cur, count, nxt, lvl + k + 1);
        // lanes take whole split edges (tree_groups): k - 1 per set
        int max_group = 1;
        while (max_group < 32 && max_group < k - 1) max_group <<= 1;
        int G = 2;
        while (G < max_group && (uint64_t)count * (uint64_t)G < (uint64_t)target_lanes) G <<= 1;
        G = G <= 2 ? 2 : (G <= 8 ? 8 : 32);
        if (G == 2) {
            tree_groups<2, MASKED, kPipe>(d, gwarp * 16, nwarps * 16, cur, count, k, memo, memo_left, pairs);
        } else if (G == 8) {
            tree_groups<8, MASKED, kPipe>(d, gwarp * 4, nwarps * 4, cur, count, k, memo, memo_left, pairs);
        } else {
            tree_groups<32, MASKED, kPipe>(d, gwarp, nwarps, cur, count, k, memo, memo_left, pairs);
        }
        if (!grid_barrier<true>(bar, epoch, max_polls)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t full = (n == 32) ? 0xFFFFFFFFu : ((1u << n) - 1u);
        extract_plan(memo, memo_left, full, d.h->hz_packed ? kWidthMask : 0xFFFFFFFFu, tree, tree_n);
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

// ---------------------------------------------------------------------------
// k_ovf_chunks / k_ovf_finalize: large sets split over all warps
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kBlock, 3) k_ovf_chunks(const uint32_t *__restrict__ blob, uint32_t blob_words, int k,
                                                       LevelCounters *__restrict__ lc, const float4 *__restrict__ memo,
                                                       const uint32_t *__restrict__ ovf_set,
                                                       const uint32_t *__restrict__ ovf_P,
                                                       const uint32_t *__restrict__ ovf_off,
                                                       unsigned long long *__restrict__ ovf_key,
                                                       unsigned long long *__restrict__ ovf_first,
                                                       GlobalCounters *__restrict__ glob, int ccc) {
    const unsigned long long packed = lc->ovf_packed;
    const uint32_t n_ovf = (uint32_t)(packed >> 40);
    const uint32_t n_chunks = (uint32_t)(packed & 0xFFFFFFFFFFull);
    if (n_ovf == 0) return;
    extern __shared__ __align__(16) uint32_t sm[];
    load_blob_to_smem(blob, blob_words, sm);
    const DevInfoView d = make_view(sm);
    const uint32_t *adj = d.h->adj;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *q = sm + ((blob_words + 3u) & ~3u) + warp * kQueueWords;
    unsigned long long pairs = 0;
    Blocks B;
    B.nb = 0;
    uint32_t cur_idx = kFull;
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&lc->chunk_next, 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= n_chunks) break;
        // largest idx with ovf_off[idx] <= c (ovf_off increases with idx)
        uint32_t lo_i = 0, hi_i = n_ovf - 1;
        while (lo_i < hi_i) {
            uint32_t mid = (lo_i + hi_i + 1) >> 1;
            if (ovf_off[mid] <= c) lo_i = mid;
            else hi_i = mid - 1;
        }
        const uint32_t idx = lo_i;
        const uint32_t S = ovf_set[idx];
        const uint32_t P = ovf_P[idx];
        if (MODE == kModeMpdp && idx != cur_idx) find_blocks(S, adj, B);
        cur_idx = idx;
        const uint32_t W = ovf_work(MODE, P);
        uint32_t lo = (c - ovf_off[idx]) * kChunk;
        uint32_t hi = lo + kChunk < W ? lo + kChunk : W;
        LaneBest best;
        best.init();
        if constexpr (MODE == kModeDpsub) eval_range_dpsub(d, adj, S, P, lo, hi, memo, q, ccc != 0, best);
        else eval_range<MODE>(d, adj, S, B, lo, hi, memo, q, ccc != 0, best);
        unsigned long long mk, fk;
        warp_winner(best, mk, fk);
        if (lane == 0) {
            if (mk != ~0ull) atomicMin(&ovf_key[idx], mk);
            atomicMin(&ovf_first[idx], fk);
        }
        pairs += best.n_valid;
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

template <int MODE>
__global__ void __launch_bounds__(kBlock) k_ovf_finalize(const uint32_t *__restrict__ blob, uint32_t blob_words,
                                                         LevelCounters *__restrict__ lc, float4 *__restrict__ memo,
                                                         uint32_t *__restrict__ memo_left,
                                                         const uint32_t *__restrict__ ovf_set,
                                                         const unsigned long long *__restrict__ ovf_key,
                                                         const unsigned long long *__restrict__ ovf_first) {
    const uint32_t n_ovf = (uint32_t)(lc->ovf_packed >> 40);
    if (n_ovf == 0) return;
    extern __shared__ __align__(16) uint32_t sm[];
    load_blob_to_smem(blob, blob_words, sm);
    const DevInfoView d = make_view(sm);
    const uint32_t *adj = d.h->adj;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n_ovf; idx += gridDim.x * blockDim.x) {
        const uint32_t S = ovf_set[idx];
        const unsigned long long first = ovf_first[idx];
        const uint32_t p = (first & 1ull) ? (uint32_t)(first >> 1) : (uint32_t)ovf_key[idx];
        uint32_t L, R;
        if (MODE == kModeDpsub || d.h->index_order) {
            L = pdep32(p + 1u, S);
            R = S ^ L;
        } else {
            Blocks B;
            find_blocks(S, adj, B);
            int b = 0;
            while (b + 1 < B.nb && B.prefix[b + 1] <= p) b++;
            uint32_t blk = B.mask[b];
            uint32_t lb = pdep32(p - B.prefix[b] + 1u, blk);
            uint32_t rb = blk ^ lb;
            L = grow(lowest(lb), S & ~rb, adj);
            R = grow(lowest(rb), S & ~lb, adj);
        }
        RelVal l = load_rel(memo, L, d.h->hz_packed), r = load_rel(memo, R, d.h->hz_packed);
        RelVal out = join_eval(d, L, l, R, r);
        memo_write(*d.h, memo, memo_left, S, out, L);
    }
}

// ---------------------------------------------------------------------------
// DPsize (gpuqo_cpu_dpsize.cu:28-96 with gpuqo_cpu_sequential.cu:28-58): for
// join size k = 2..n, left size m = k-1 down to 1, every relation set L of the
// level-m list and R of the level-(k-m) list, in list order, a disjoint and
// connected pair (L, R) is costed as L joining R; the set L + R keeps its
// first strict minimum (a NaN cost first found is kept), and is appended to
// the level-k list when it is first produced.  The level-1 list is the
// iteration order of the reference's unordered_map memo after the base
// relations are inserted (dpsize_level1_places); later lists are in
// discovery order.
//
// Here every connected k-set S is costed on its own (one warp, the valid
// splits of S from the biconnected-block enumeration), with each split keyed
// by its place in that loop: G = off[|L|] + pos[L], off[m] = the sizes of
// levels m+1 .. k-1 (larger left sides first), pos[] the position of a set in
// its level list.  The lexicographic minimum of (cost, G) is the reference's
// first strict minimum.  S is first produced by its split of smallest
// (G, pos[R]); that split always has |L| = k-1 (every connected set has a
// relation whose removal leaves it connected), so S's discovery key is
// (pos[L*], pos[v*]) with v* the relation outside L*.  The level-k list order
// follows from the keys without a sort: the sets discovered from one L* are
// L* + v for different relations v, so one 32-bit mask per level-(k-1) set
// collects the pos[v] of its discoveries, an exclusive scan of the mask
// popcounts gives each L*'s first place, and a set's place is that plus the
// number of lower bits in its L*'s mask.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_dpsize_eval(const uint32_t *__restrict__ blob, uint32_t blob_words,
                                                        int k, const uint32_t *__restrict__ sets,
                                                        const LevelCounters *__restrict__ lvl,
                                                        float4 *__restrict__ memo, uint32_t *__restrict__ memo_left,
                                                        const uint32_t *__restrict__ pos,
                                                        unsigned long long *__restrict__ disc,
                                                        uint32_t *__restrict__ bmask,
                                                        GlobalCounters *__restrict__ glob) {
    const uint32_t count = __ldcg(&lvl[k].n_sets);
    if (count == 0u) return;
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t off[33];
    load_blob_to_smem(blob, blob_words, sm);
    const DevInfoView d = make_view(sm);
    const uint32_t *adj = d.h->adj;
    if (threadIdx.x == 0) {
        // off[m] = sizes of the levels m+1 .. k-1; level 1 holds the n relations
        uint32_t acc = 0u;
        for (int m = k - 1; m >= 1; m--) {
            off[m] = acc;
            acc += (m == 1) ? (uint32_t)d.h->n : __ldcg(&lvl[m].n_sets);
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    unsigned long long pairs = 0;
    Blocks B;
    CycleCache cc;
    for (uint32_t i = blockIdx.x * kWarpsPerBlock + warp; i < count; i += nwarps) {
        const uint32_t S = __ldcg(sets + i);
        find_blocks(S, adj, B);
        const uint32_t P = B.etotal;
        LaneBest best;
        best.init();
        unsigned long long dmin = ~0ull;
        int b = 0;
        for (uint32_t c = (uint32_t)lane; c < P; c += 32u) {
            uint32_t L, R, key;
            if (!mpdp_candidate(S, B, adj, c, b, L, R, key, cc)) continue;
            const uint32_t g = off[__popc(L)] + __ldcg(pos + L);
            const unsigned long long dk = ((unsigned long long)g << 32) | __ldcg(pos + R);
            if (dk < dmin) dmin = dk;
            const RelVal l = load_rel(memo, L, d.h->hz_packed), r = load_rel(memo, R, d.h->hz_packed);
            best_update(best, g, L, join_eval(d, L, l, R, r));
        }
        unsigned long long mk, fk;
        const WarpWinner w = warp_winner(best, mk, fk);
        if (w.is_writer) {
            if (w.use_nan) memo_write(*d.h, memo, memo_left, S, best.nan_val, best.nan_left);
            else memo_write(*d.h, memo, memo_left, S, best.val, best.left);
        }
        const uint32_t dh = __reduce_min_sync(kFull, (uint32_t)(dmin >> 32));
        const uint32_t dl = __reduce_min_sync(kFull, (uint32_t)(dmin >> 32) == dh ? (uint32_t)dmin : kFull);
        if (lane == 0) {
            disc[i] = ((unsigned long long)dh << 32) | dl;
            atomicOr(bmask + dh, 1u << dl);
        }
        pairs += best.n_valid;
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

constexpr uint32_t kScanTile = kBlock * 4;   // mask words per block of the place scan

// block b: the popcount total of bmask[b * kScanTile ..) (entries < level k-1's size)
__global__ void __launch_bounds__(kBlock) k_dpsize_scan_tiles(const uint32_t *__restrict__ bmask,
                                                              const LevelCounters *__restrict__ lvl, int km1, int n,
                                                              uint32_t *__restrict__ tile_sum) {
    const uint32_t cnt = km1 == 1 ? (uint32_t)n : __ldcg(&lvl[km1].n_sets);
    const uint32_t base = blockIdx.x * kScanTile;
    if (base >= cnt) return;
    uint32_t v = 0u;
    for (uint32_t j = threadIdx.x; j < kScanTile; j += kBlock)
        if (base + j < cnt) v += (uint32_t)__popc(__ldcg(bmask + base + j));
    v = __reduce_add_sync(kFull, v);
    __shared__ uint32_t ws[kWarpsPerBlock];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0u;
        for (int w = 0; w < kWarpsPerBlock; w++) t += ws[w];
        tile_sum[blockIdx.x] = t;
    }
}

// one block: exclusive scan of the tile totals, in place
__global__ void __launch_bounds__(kBlock) k_dpsize_scan_top(uint32_t *__restrict__ tile_sum,
                                                            const LevelCounters *__restrict__ lvl, int km1, int n) {
    const uint32_t cnt = km1 == 1 ? (uint32_t)n : __ldcg(&lvl[km1].n_sets);
    const uint32_t tiles = (cnt + kScanTile - 1u) / kScanTile;
    __shared__ uint32_t carry;
    __shared__ uint32_t ws[kWarpsPerBlock];
    if (threadIdx.x == 0) carry = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < tiles; base += kBlock) {
        const uint32_t idx = base + threadIdx.x;
        const uint32_t v = idx < tiles ? tile_sum[idx] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) ws[warp] = incl;
        __syncthreads();
        uint32_t wpre = 0u, total = 0u;
        for (int w = 0; w < kWarpsPerBlock; w++) {
            if (w < warp) wpre += ws[w];
            total += ws[w];
        }
        if (idx < tiles) tile_sum[idx] = carry + wpre + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

// block b: bstart[j] = exclusive prefix of the mask popcounts for the masks j
// of tile b (the tile's offset from k_dpsize_scan_top plus the popcounts of
// the tile's earlier masks); each thread takes 4 consecutive masks
__global__ void __launch_bounds__(kBlock) k_dpsize_scan_fill(const uint32_t *__restrict__ bmask,
                                                             const LevelCounters *__restrict__ lvl, int km1, int n,
                                                             const uint32_t *__restrict__ tile_sum,
                                                             uint32_t *__restrict__ bstart) {
    const uint32_t cnt = km1 == 1 ? (uint32_t)n : __ldcg(&lvl[km1].n_sets);
    const uint32_t base = blockIdx.x * kScanTile;
    if (base >= cnt) return;
    const uint32_t j0 = base + threadIdx.x * 4u;
    uint32_t c[4], tot = 0u;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        c[q] = (j0 + q < cnt) ? (uint32_t)__popc(__ldcg(bmask + j0 + q)) : 0u;
        tot += c[q];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    __shared__ uint32_t ws[kWarpsPerBlock];
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    uint32_t run = __ldcg(tile_sum + blockIdx.x) + incl - tot;
    for (int w = 0; w < warp; w++) run += ws[w];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (j0 + q < cnt) bstart[j0 + q] = run;
        run += c[q];
    }
}

// every set of level k: its place in the level-k list
__global__ void __launch_bounds__(kBlock) k_dpsize_place(const uint32_t *__restrict__ sets,
                                                         const LevelCounters *__restrict__ lvl, int k,
                                                         const unsigned long long *__restrict__ disc,
                                                         const uint32_t *__restrict__ bmask,
                                                         const uint32_t *__restrict__ bstart,
                                                         uint32_t *__restrict__ pos) {
    const uint32_t count = __ldcg(&lvl[k].n_sets);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const unsigned long long dk = __ldcg(disc + i);
        const uint32_t bl = (uint32_t)(dk >> 32), v = (uint32_t)dk;
        pos[__ldcg(sets + i)] = __ldcg(bstart + bl) + (uint32_t)__popc(__ldcg(bmask + bl) & ((1u << v) - 1u));
    }
}

// the masks of the level-(k-1) sets, cleared once every place is read
__global__ void __launch_bounds__(kBlock) k_dpsize_clear(uint32_t *__restrict__ bmask,
                                                         const LevelCounters *__restrict__ lvl, int km1, int n) {
    const uint32_t cnt = km1 == 1 ? (uint32_t)n : __ldcg(&lvl[km1].n_sets);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) bmask[j] = 0u;
}

// the level-1 list: pos[1 << i] = place of relation i
__global__ void k_dpsize_init(uint32_t *__restrict__ pos, const uint32_t *__restrict__ level1, int n) {
    const int i = threadIdx.x;
    if (i < n) pos[1u << i] = level1[i];
}

// ---------------------------------------------------------------------------
// base relations and plan extraction
// ---------------------------------------------------------------------------
__global__ void k_init_base(const uint32_t *__restrict__ blob, float4 *__restrict__ memo,
                            uint32_t *__restrict__ memo_left) {
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob);
    int i = threadIdx.x;
    if (i < h->n) {
        // gpuqo_cpu_sequential.cu:80-92: base relation memo entries
        memo[1u << i] = base_entry(*h, i);
        memo_left[1u << i] = 0u;
    }
}

__global__ void k_extract(const float4 *__restrict__ memo, const uint32_t *__restrict__ memo_left, uint32_t full,
                          const uint32_t *__restrict__ blob, TreeNode *__restrict__ out, int *__restrict__ n_out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t wmask = reinterpret_cast<const DevHeader *>(blob)->hz_packed ? kWidthMask : 0xFFFFFFFFu;
    // iterative preorder walk; node i's children are appended after it
    int n = 0;
    uint32_t stack_set[64];
    int stack_parent[64];
    int stack_side[64];
    int sp = 0;
    stack_set[sp] = full;
    stack_parent[sp] = -1;
    stack_side[sp] = 0;
    sp++;
    while (sp > 0 && n < 64) {
        sp--;
        uint32_t s = stack_set[sp];
        int parent = stack_parent[sp], side = stack_side[sp];
        float4 v = memo[s];
        TreeNode t;
        t.set = s;
        t.left = -1;
        t.right = -1;
        t.rows = v.x;
        t.startup = v.y;
        t.total = v.z;
        t.width = (int)(__float_as_uint(v.w) & wmask);
        int me = n++;
        out[me] = t;
        if (parent >= 0) {
            if (side == 0) out[parent].left = me;
            else out[parent].right = me;
        }
        uint32_t l = memo_left[s] & s;
        if (__popc(s) > 1 && l != 0u && l != s && sp + 2 <= 64) {
            uint32_t r = s ^ l;
            stack_set[sp] = r;
            stack_parent[sp] = me;
            stack_side[sp] = 1;
            sp++;
            stack_set[sp] = l;
            stack_parent[sp] = me;
            stack_side[sp] = 0;
            sp++;
        }
    }
    *n_out = n;
}

// ---------------------------------------------------------------------------
// host engine
// ---------------------------------------------------------------------------
static uint64_t binom64(int n, int k) {
    if (k < 0 || k > n) return 0;
    uint64_t r = 1;
    for (int i = 1; i <= k; i++) r = r * (uint64_t)(n - k + i) / (uint64_t)i;
    return r;
}

static uint64_t max_level_sets(int n) {
    uint64_t m = 1;
    for (int k = 0; k <= n; k++) m = std::max(m, binom64(n, k));
    return m;
}

uint64_t engine_bytes_needed(int n) {
    uint64_t memo = (1ull << n) * (sizeof(float4) + sizeof(uint32_t));
    uint64_t lv = max_level_sets(n) * (4ull * 4 + 8ull * 2);
    return memo + lv + (1u << 20);
}

// a failed allocation is GPUQO_B200_ERR_NOMEM (it leaves no sticky error:
// the next call may succeed), any other failure GPUQO_B200_ERR_CUDA
#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            if (e_ == cudaErrorMemoryAllocation) {                                        \
                cudaGetLastError();                                                       \
                return GPUQO_B200_ERR_NOMEM;                                              \
            }                                                                             \
            return GPUQO_B200_ERR_CUDA;                                                   \
        }                                                                                 \
    } while (0)

// gpuqo_b200_device_memory_mb: when > 0, a DP whose arena would need more
// device memory than this is refused with GPUQO_B200_ERR_NOMEM before any
// allocation (the engines keep what they hold, so later calls are unaffected)
static int over_budget(uint64_t bytes, const char *what, std::string &err) {
    const int mb = gpuqo_b200_device_memory_mb;
    if (mb <= 0 || bytes <= ((uint64_t)mb << 20)) return 0;
    err = std::string(what) + " needs " + std::to_string(bytes >> 20) + " MB of device memory; " +
          "gpuqo_b200_device_memory_mb allows " + std::to_string(mb);
    return GPUQO_B200_ERR_NOMEM;
}

struct GraphKey {
    int n, mode, ccc, profile;
    bool operator<(const GraphKey &o) const {
        if (n != o.n) return n < o.n;
        if (mode != o.mode) return mode < o.mode;
        if (ccc != o.ccc) return ccc < o.ccc;
        return profile < o.profile;
    }
};

// Parameters the autotuner (engine_autotune) measures; these defaults apply
// until it runs.  Neither changes a plan, only which kernel variant runs.
struct Tuning {
    // tree queries with up to this many connected sets per level run
    // k_dp_tree<2>, those with more than single_wide_level_sets k_dp_tree<4>
    double single_narrow_level_sets = 16384.0;
    double single_wide_level_sets = 1e30;
    double batch_single_sets = double(1u << 20);   // a batch hands larger tree queries to k_dp_tree
    bool tuned = false;
};
constexpr int kMaxDevices = 64;
static Tuning g_tuning[kMaxDevices];            // per device, guarded by g_dev_mu

static double tree_connected_sets(const DevHeader *h);

// cpu_dpsize's level-1 list (gpuqo_cpu_dpsize.cu:43-48 after
// gpuqo_cpu_sequential.cu:73-84): the iteration order of its unordered_map
// memo once base relation i (key 2^(i+1), whose hash is the key itself) has
// been inserted for i = 0 .. n-1.  The same standard-library container,
// filled the same way, gives the same order; place[i] = position of relation i.
static std::vector<uint32_t> dpsize_level1_places(int n) {
    std::unordered_map<uint32_t, int> m;
    for (int i = 0; i < n; i++) m.insert(std::make_pair(1u << (i + 1), i));
    std::vector<uint32_t> place((size_t)n, 0u);
    uint32_t p = 0;
    for (const auto &kv : m) place[(size_t)kv.second] = p++;
    return place;
}

// Per-run control words of the single-query engine, contiguous so that one
// memset clears the counters and one copy brings everything back.
struct EngineCtl {
    LevelCounters lvl[33];
    GlobalCounters glob;
    unsigned bar[4];                   // grid barrier of k_dp_tree: arrivals, -, error flag
    int tree_n;
    int pad;
    TreeNode tree[64];
};
constexpr size_t kCtlClearBytes = offsetof(EngineCtl, pad);   // lvl .. tree_n

class Engine {
public:
    int device = -1;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    DevArena a;
    int cap_n = -1;                    // arena sized for this many relations
    uint64_t cap_sets = 0;
    uint32_t blob_cap_words = 0;
    uint32_t *h_blob = nullptr;        // pinned staging
    uint32_t h_level1[32];             // staging of the DPsize level-1 list (copied before each launch)
    EngineCtl *d_ctl = nullptr;        // device control words (a.lvl, a.glob, a.bar, a.tree_n, a.tree point here)
    EngineCtl *h_ctl = nullptr;        // pinned copy
    TreeNode *h_tree = nullptr;        // views into h_ctl
    int *h_tree_n = nullptr;
    GlobalCounters *h_glob = nullptr;
    LevelCounters *h_lvl = nullptr;
    std::map<GraphKey, cudaGraphExec_t> graphs;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> kev;      // per-level eval events (profile mode)
    int n_kernels = 0;                 // kernels per DP run
    unsigned *h_bar = nullptr;         // pinned copy of the barrier words
    std::map<size_t, int> coop_blocks; // (dynamic shared bytes, variant) -> co-resident blocks of k_dp_tree (0: none)
    int force_minb = 0;                // autotuner: run this k_dp_tree variant (2, 3 or 4); 0 = by the tuning record
    bool coop_off = false;             // cooperative launch refused on this device
    bool barrier_timed_out = false;    // a grid barrier of k_dp_tree gave up: per-level launches until reset
    std::map<GraphKey, int> graph_kernels;
    float *flush = nullptr;            // L2 flush buffer (timing only)

    int init(std::string &err) {
        if (stream) return 0;
        CK(cudaGetDevice(&device));
        CK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        kev.resize(2 * 34);
        for (auto &e : kev) CK(cudaEventCreate(&e));
        CK(cudaMalloc(&d_ctl, sizeof(EngineCtl)));
        CK(cudaMallocHost(&h_ctl, sizeof(EngineCtl)));
        a.lvl = d_ctl->lvl;
        a.glob = &d_ctl->glob;
        a.bar = d_ctl->bar;
        a.tree_n = &d_ctl->tree_n;
        a.tree = d_ctl->tree;
        h_lvl = h_ctl->lvl;
        h_glob = &h_ctl->glob;
        h_bar = h_ctl->bar;
        h_tree_n = &h_ctl->tree_n;
        h_tree = h_ctl->tree;
        CK(cudaMalloc(&a.binom, 33 * 33 * sizeof(uint32_t)));
        std::vector<uint32_t> bt(33 * 33, 0);
        for (int i = 0; i <= 32; i++)
            for (int j = 0; j <= 32; j++) {
                uint64_t v = binom64(i, j);
                bt[i * 33 + j] = v > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)v;
            }
        CK(cudaMemcpy(a.binom, bt.data(), bt.size() * 4, cudaMemcpyHostToDevice));
        return 0;
    }

    void drop_graphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }

    int ensure(int n, uint32_t blob_words, std::string &err) {
        if (blob_words > blob_cap_words) {
            drop_graphs();
            if (a.blob) cudaFree(a.blob);
            if (h_blob) cudaFreeHost(h_blob);
            uint32_t cap = std::max<uint32_t>((blob_words + 511u) & ~511u, 16384u);
            CK(cudaMalloc(&a.blob, cap * 4));
            CK(cudaMallocHost(&h_blob, cap * 4));
            blob_cap_words = cap;
        }
        // the budget bounds what one DP needs, whatever the engine already holds
        if (int rc = over_budget(engine_bytes_needed(n), "the exact DP's dense memo and level lists", err)) return rc;
        if (n <= cap_n) return 0;
        drop_graphs();
        cudaFree(a.memo);
        cudaFree(a.memo_left);
        cudaFree(a.sets);
        cudaFree(a.sets2);
        cudaFree(a.seen);
        cudaFree(a.ovf_set);
        cudaFree(a.ovf_P);
        cudaFree(a.ovf_off);
        cudaFree(a.ovf_key);
        cudaFree(a.ovf_first);
        a.memo = nullptr;
        cap_n = -1;
        uint64_t slots = 1ull << n;
        uint64_t ms = max_level_sets(n);
        CK(cudaMalloc(&a.memo, slots * sizeof(float4)));
        CK(cudaMalloc(&a.memo_left, slots * sizeof(uint32_t)));
        CK(cudaMalloc(&a.sets, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.sets2, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.seen, std::max<uint64_t>(slots / 8, 4)));
        CK(cudaMalloc(&a.ovf_set, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.ovf_P, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.ovf_off, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.ovf_key, ms * sizeof(unsigned long long)));
        CK(cudaMalloc(&a.ovf_first, ms * sizeof(unsigned long long)));
        cap_n = n;
        cap_sets = ms;
        return 0;
    }

    int dpsize_cap_n = -1;             // DPsize buffers sized for this many relations

    int ensure_dpsize(int n, std::string &err) {
        const uint64_t ms = max_level_sets(n);
        const uint64_t tiles = ms / kScanTile + 2;
        if (int rc = over_budget(engine_bytes_needed(n) + (1ull << n) * 4 + ms * 16 + tiles * 4,
                                 "DPsize's dense memo, level lists and place arrays", err))
            return rc;
        if (n <= dpsize_cap_n) return 0;
        drop_graphs();
        cudaFree(a.pos);
        cudaFree(a.bmask);
        cudaFree(a.bstart);
        cudaFree(a.tile_sum);
        cudaFree(a.disc);
        a.pos = a.bmask = a.bstart = a.tile_sum = nullptr;
        a.disc = nullptr;
        dpsize_cap_n = -1;
        CK(cudaMalloc(&a.pos, (1ull << n) * sizeof(uint32_t)));
        CK(cudaMalloc(&a.bmask, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.bstart, ms * sizeof(uint32_t)));
        CK(cudaMalloc(&a.tile_sum, tiles * sizeof(uint32_t)));
        CK(cudaMalloc(&a.disc, ms * sizeof(unsigned long long)));
        if (!a.level1) CK(cudaMalloc(&a.level1, 32 * sizeof(uint32_t)));
        dpsize_cap_n = n;
        return 0;
    }

    // DPsize of n relations on `stream` (see k_dpsize_eval)
    int enqueue_dpsize(int n, uint32_t blob_words, std::string &err) {
        const size_t smem = eval_smem(blob_words);
        CK(cudaMemsetAsync(d_ctl, 0, kCtlClearBytes, stream));
        CK(cudaMemsetAsync(a.seen, 0, std::max<uint64_t>((1ull << n) / 8, 4), stream));
        CK(cudaMemsetAsync(a.bmask, 0, max_level_sets(n) * sizeof(uint32_t), stream));
        n_kernels = 0;
        k_init_base<<<1, 32, 0, stream>>>(a.blob, a.memo, a.memo_left);
        k_dpsize_init<<<1, 32, 0, stream>>>(a.pos, a.level1, n);
        n_kernels += 2;
        for (int k = 2; k <= n; k++) {
            const uint64_t total = binom64(n, k);
            uint64_t threads = std::min<uint64_t>((uint64_t)sm_count * 8 * kBlock, (total + 3) / 4);
            threads = std::max<uint64_t>(threads, 32);
            const uint32_t per_thread = (uint32_t)((total + threads - 1) / threads);
            const uint32_t fblocks =
                (uint32_t)((total + (uint64_t)per_thread * kBlock - 1) / ((uint64_t)per_thread * kBlock));
            uint32_t *cur_sets = (k & 1) ? a.sets2 : a.sets;
            const uint32_t *prev_sets = (k & 1) ? a.sets : a.sets2;
            k_level_sets<<<fblocks, kBlock, 0, stream>>>(a.blob, a.binom, n, k, total, per_thread, prev_sets,
                                                         a.lvl + (k - 1), a.seen, cur_sets, a.lvl + k);
            const int eblocks =
                (int)std::min<uint64_t>((uint64_t)sm_count * 4, (total + kWarpsPerBlock - 1) / kWarpsPerBlock);
            CK(cudaEventRecordWithFlags(kev[2 * k], stream, cudaEventRecordExternal));
            k_dpsize_eval<<<eblocks, kBlock, smem, stream>>>(a.blob, blob_words, k, cur_sets, a.lvl, a.memo,
                                                             a.memo_left, a.pos, a.disc, a.bmask, a.glob);
            CK(cudaEventRecordWithFlags(kev[2 * k + 1], stream, cudaEventRecordExternal));
            // places of the level-k sets from the masks of the level-(k-1) sets
            const uint64_t prev_total = binom64(n, k - 1);
            const uint32_t tiles = (uint32_t)((prev_total + kScanTile - 1) / kScanTile);
            k_dpsize_scan_tiles<<<tiles, kBlock, 0, stream>>>(a.bmask, a.lvl, k - 1, n, a.tile_sum);
            k_dpsize_scan_top<<<1, kBlock, 0, stream>>>(a.tile_sum, a.lvl, k - 1, n);
            k_dpsize_scan_fill<<<tiles, kBlock, 0, stream>>>(a.bmask, a.lvl, k - 1, n, a.tile_sum, a.bstart);
            const uint32_t pblocks = (uint32_t)std::min<uint64_t>((uint64_t)sm_count * 8, (total + kBlock - 1) / kBlock);
            k_dpsize_place<<<pblocks, kBlock, 0, stream>>>(cur_sets, a.lvl, k, a.disc, a.bmask, a.bstart, a.pos);
            const uint32_t cblocks =
                (uint32_t)std::min<uint64_t>((uint64_t)sm_count * 8, (prev_total + kBlock - 1) / kBlock);
            k_dpsize_clear<<<cblocks, kBlock, 0, stream>>>(a.bmask, a.lvl, k - 1, n);
            n_kernels += 7;
        }
        const uint32_t full = (n == 32) ? 0xFFFFFFFFu : ((1u << n) - 1u);
        k_extract<<<1, 32, 0, stream>>>(a.memo, a.memo_left, full, a.blob, a.tree, a.tree_n);
        n_kernels++;
        return 0;
    }

    size_t eval_smem(uint32_t blob_words) const {
        return (size_t)(((blob_words + 3u) & ~3u) + kWarpsPerBlock * kQueueWords) * 4u;
    }

    // Enqueues the whole DP for n relations on `stream`.
    int enqueue(int n, DpMode mode, bool ccc, bool profile, uint32_t blob_words, std::string &err) {
        if (mode == kModeDpsize) return enqueue_dpsize(n, blob_words, err);
        const size_t smem = eval_smem(blob_words);
        const uint32_t max_block = reinterpret_cast<const DevHeader *>(h_blob)->max_block;
        const bool tree_mode = reinterpret_cast<const DevHeader *>(h_blob)->tree_mode != 0u;
        const int eval_max_blocks = sm_count * 4;
        CK(cudaMemsetAsync(d_ctl, 0, kCtlClearBytes, stream));
        CK(cudaMemsetAsync(a.seen, 0, std::max<uint64_t>((1ull << n) / 8, 4), stream));
        n_kernels = 0;
        k_init_base<<<1, 32, 0, stream>>>(a.blob, a.memo, a.memo_left);
        n_kernels++;
        for (int k = 2; k <= n; k++) {
            uint64_t total = binom64(n, k);
            uint64_t threads_cap = (uint64_t)sm_count * 8 * kBlock;
            uint64_t threads = std::min<uint64_t>(threads_cap, (total + 3) / 4);
            threads = std::max<uint64_t>(threads, 32);
            uint32_t per_thread = (uint32_t)((total + threads - 1) / threads);
            uint32_t fblocks = (uint32_t)((total + (uint64_t)per_thread * kBlock - 1) / ((uint64_t)per_thread * kBlock));
            LevelCounters *lc = a.lvl + k;
            uint32_t *cur_sets = (k & 1) ? a.sets2 : a.sets;
            const uint32_t *prev_sets = (k & 1) ? a.sets : a.sets2;
            k_level_sets<<<fblocks, kBlock, 0, stream>>>(a.blob, a.binom, n, k, total, per_thread, prev_sets,
                                                         a.lvl + (k - 1), a.seen, cur_sets, lc);
            n_kernels += 2;
            int eblocks = (int)std::min<uint64_t>((uint64_t)eval_max_blocks, (total + kWarpsPerBlock - 1) / kWarpsPerBlock);
            CK(cudaEventRecordWithFlags(kev[2 * k], stream, cudaEventRecordExternal));
            if (mode == kModeDpsub) {
                k_eval<kModeDpsub><<<eblocks, kBlock, smem, stream>>>(a.blob, blob_words, k, cur_sets, lc, a.memo,
                                                                      a.memo_left, a.ovf_set, a.ovf_P, a.ovf_off,
                                                                      a.ovf_key, a.ovf_first, a.glob, ccc);
            } else {
                // max useful group: pairs of a k-set are at least 2(k-1)
                int max_group = 1;
                while (max_group < 32 && max_group < 2 * (k - 1)) max_group <<= 1;
                const uint32_t target_lanes = (uint32_t)sm_count * 24u * 32u;
                int mblocks = (int)std::min<uint64_t>((uint64_t)sm_count * 4, (total * 32 + kBlock - 1) / kBlock);
                if (tree_mode) {
                    // the tree kernel's lanes take split edges: k - 1 per set
                    int max_edge_group = 1;
                    while (max_edge_group < 32 && max_edge_group < k - 1) max_edge_group <<= 1;
                    k_eval_tree<<<mblocks, kBlock, smem, stream>>>(a.blob, blob_words, k, cur_sets, lc, a.memo,
                                                                   a.memo_left, a.glob, target_lanes, max_edge_group);
                } else {
                    k_eval_mpdp<<<mblocks, kBlock, smem, stream>>>(a.blob, blob_words, cur_sets, lc, a.memo,
                                                                   a.memo_left, a.ovf_set, a.ovf_P, a.ovf_off,
                                                                   a.ovf_key, a.ovf_first, a.glob, target_lanes,
                                                                   max_group);
                }
            }
            CK(cudaEventRecordWithFlags(kev[2 * k + 1], stream, cudaEventRecordExternal));
            bool may_overflow;
            if (mode == kModeDpsub) {
                may_overflow = ((1ull << k) - 2ull) > kOvfLimit;
            } else {
                // sum over blocks of 2^|b| - 2 with sum(|b| - 1) = k - 1 and
                // |b| <= the query graph's largest block
                int bmax = std::min<int>(std::max<int>((int)max_block, 2), k);
                uint64_t nblk = (uint64_t)(k - 1 + bmax - 2) / (uint64_t)(bmax - 1);
                may_overflow = nblk * ((1ull << bmax) - 2ull) > kOvfLimit;
            }
            if (may_overflow) {
                n_kernels += 2;
                int oblocks = sm_count * 4;
                if (mode == kModeDpsub) {
                    k_ovf_chunks<kModeDpsub><<<oblocks, kBlock, smem, stream>>>(
                        a.blob, blob_words, k, lc, a.memo, a.ovf_set, a.ovf_P, a.ovf_off, a.ovf_key, a.ovf_first,
                        a.glob, ccc);
                    k_ovf_finalize<kModeDpsub><<<sm_count, kBlock, smem, stream>>>(
                        a.blob, blob_words, lc, a.memo, a.memo_left, a.ovf_set, a.ovf_key, a.ovf_first);
                } else {
                    k_ovf_chunks<kModeMpdp><<<oblocks, kBlock, smem, stream>>>(
                        a.blob, blob_words, k, lc, a.memo, a.ovf_set, a.ovf_P, a.ovf_off, a.ovf_key, a.ovf_first,
                        a.glob, ccc);
                    k_ovf_finalize<kModeMpdp><<<sm_count, kBlock, smem, stream>>>(
                        a.blob, blob_words, lc, a.memo, a.memo_left, a.ovf_set, a.ovf_key, a.ovf_first);
                }
            }
        }
        uint32_t full = (n == 32) ? 0xFFFFFFFFu : ((1u << n) - 1u);
        k_extract<<<1, 32, 0, stream>>>(a.memo, a.memo_left, full, a.blob, a.tree, a.tree_n);
        n_kernels++;
        return 0;
    }

    int download(std::string &err) {
        CK(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream));
        return 0;
    }

    // The whole tree-mode MPDP as one cooperative launch (k_dp_tree).  Returns
    // 0 and sets launched when the kernel was started.
    int launch_persistent(int n, uint32_t words, bool &launched, std::string &err) {
        launched = false;
        const size_t smem = (size_t)(((words + 3u) & ~3u) + 33 * 33 + 3 + kWarpsPerBlock * 64) * 4u;
        if (coop_off) return 0;
        int minb = force_minb;
        if (minb == 0) {
            const double per_level = tree_connected_sets(reinterpret_cast<const DevHeader *>(h_blob)) / n;
            const Tuning &tu = g_tuning[device];
            minb = per_level <= tu.single_narrow_level_sets ? 2 : (per_level > tu.single_wide_level_sets ? 4 : 3);
        }
        const bool masked = reinterpret_cast<const DevHeader *>(h_blob)->ec_masked != 0u;
        const void *fn = masked ? (minb == 4   ? (const void *)k_dp_tree<4, true>
                                   : minb == 2 ? (const void *)k_dp_tree<2, true>
                                               : (const void *)k_dp_tree<3, true>)
                                : (minb == 4   ? (const void *)k_dp_tree<4, false>
                                   : minb == 2 ? (const void *)k_dp_tree<2, false>
                                               : (const void *)k_dp_tree<3, false>);
        const size_t key = smem * 16u + (size_t)minb * 2u + (masked ? 1u : 0u);
        auto cb = coop_blocks.find(key);
        if (cb == coop_blocks.end()) {
            int blocks = 0, dev_coop = 0, occ = 0;
            cudaDeviceGetAttribute(&dev_coop, cudaDevAttrCooperativeLaunch, device);
            bool ok = dev_coop != 0;
            if (ok && smem > 48 * 1024)
                ok = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess;
            if (ok) ok = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBlock, smem) == cudaSuccess;
            if (ok) blocks = occ * sm_count;
            cudaGetLastError();
            cb = coop_blocks.emplace(key, blocks).first;
        }
        const int grid = cb->second;
        if (grid <= 0) return 0;
        CK(cudaMemsetAsync(d_ctl, 0, kCtlClearBytes, stream));   // counters, barrier words, tree size
        uint32_t bwords = words;
        // group width per level: count x G covers half the resident threads
        // (measured: narrower groups, more sets in flight, shorten the levels
        // of 20- to 25-relation trees by about 8 %; a quarter or an eighth is
        // slower again)
        uint32_t target_lanes = (uint32_t)grid * (uint32_t)kBlock / 2u;
        unsigned poll_limit = (unsigned)std::max(0, gpuqo_b200_barrier_poll_limit);
        void *args[] = {&a.blob, &bwords, &a.binom, &a.memo, &a.memo_left, &a.sets, &a.sets2,
                        &a.lvl, &a.glob, &a.tree, &a.tree_n, &a.bar, &target_lanes, &poll_limit};
        cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), args, smem, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            coop_off = true;   // do not retry on this engine
            return 0;
        }
        n_kernels = 1;
        launched = true;
        return 0;
    }

    // brings the control words back (one copy) and reports whether the last
    // persistent run's grid barrier timed out; a timeout latches the engine
    // onto the per-level launches (gpuqo_b200_reset_persistent clears it), so
    // later calls do not wait for another timeout first
    int barrier_failed(bool &failed, EngineStats &st, std::string &err) {
        if (int rc = download(err)) return rc;
        CK(cudaStreamSynchronize(stream));
        failed = h_bar[2] != 0u;
        if (failed) {
            barrier_timed_out = true;
            st.barrier_timeouts++;
        }
        return 0;
    }

    // Stages the blob, makes sure the arena and the graph for (n, mode) exist.
    int prepare(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, bool profile, uint32_t &words,
                cudaGraphExec_t &exec, std::string &err) {
        if (int rc = init(err)) return rc;
        // the blob is staged in buckets of 512 words so that one captured
        // graph serves every query of the same size class
        words = ((uint32_t)blob.size() + 511u) & ~511u;
        if (int rc = ensure(n, words, err)) return rc;
        if (mode == kModeDpsize) {
            if (int rc = ensure_dpsize(n, err)) return rc;
            const std::vector<uint32_t> l1 = dpsize_level1_places(n);
            std::memcpy(h_level1, l1.data(), l1.size() * 4);
            CK(cudaMemcpyAsync(a.level1, h_level1, l1.size() * 4, cudaMemcpyHostToDevice, stream));
        }
        std::memset(h_blob, 0, words * 4);
        std::memcpy(h_blob, blob.data(), blob.size() * 4);
        const size_t smem = eval_smem(words);
        if (smem > 48 * 1024) {
            CK(cudaFuncSetAttribute(k_dpsize_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaFuncSetAttribute(k_eval<kModeDpsub>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaFuncSetAttribute(k_eval<kModeMpdp>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaFuncSetAttribute(k_ovf_chunks<kModeDpsub>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaFuncSetAttribute(k_ovf_chunks<kModeMpdp>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaFuncSetAttribute(k_ovf_finalize<kModeDpsub>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaFuncSetAttribute(k_ovf_finalize<kModeMpdp>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        }
        CK(cudaMemcpyAsync(a.blob, h_blob, words * 4, cudaMemcpyHostToDevice, stream));
        exec = nullptr;
        const uint32_t mb = reinterpret_cast<const DevHeader *>(h_blob)->max_block;
        const uint32_t tm = reinterpret_cast<const DevHeader *>(h_blob)->tree_mode;
        GraphKey key{n, ((int)mode * 64 + (int)std::min<uint32_t>(mb, 63u)) * 2 + (int)(tm != 0u), ccc ? 1 : 0,
                     (int)words};
        (void)profile;
        auto it = graphs.find(key);
        if (it != graphs.end()) {
            exec = it->second;
            n_kernels = graph_kernels[key];
            return 0;
        }
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue(n, mode, ccc, false, words, err);
        cudaGraph_t captured = nullptr;
        cudaError_t ce = cudaStreamEndCapture(stream, &captured);
        if (rc) {
            if (captured) cudaGraphDestroy(captured);
            return rc;
        }
        if (ce != cudaSuccess) {
            err = std::string("graph capture: ") + cudaGetErrorString(ce);
            return GPUQO_B200_ERR_CUDA;
        }
        CK(cudaGraphInstantiate(&exec, captured, 0));
        cudaGraphDestroy(captured);
        graphs[key] = exec;
        graph_kernels[key] = n_kernels;
        return 0;
    }

    int launch(cudaGraphExec_t exec, std::string &err) {
        CK(cudaGraphLaunch(exec, stream));
        return 0;
    }

    // evaluate-kernel time of the last replay, from the per-level event
    // nodes captured in the graph
    int read_eval_events(int n, EngineStats &st, std::string &err) {
        for (int k = 2; k <= n; k++) {
            float kms = 0.f;
            CK(cudaEventElapsedTime(&kms, kev[2 * k], kev[2 * k + 1]));
            st.eval_kernel_ms += kms;
            st.eval_kernel_launches++;
        }
        return 0;
    }

    // Copies the plan and counters back and fills nodes / stats.
    int finish(int n, bool profile, std::vector<TreeNode> &nodes, EngineStats &st, std::string &err,
               bool downloaded = false) {
        if (!downloaded)
            if (int rc = download(err)) return rc;
        CK(cudaStreamSynchronize(stream));
        CK(cudaGetLastError());
        if (profile)
            if (int rc = read_eval_events(n, st, err)) return rc;
        int nn = *h_tree_n;
        if (nn != 2 * n - 1) {
            err = "plan extraction produced " + std::to_string(nn) + " nodes for " + std::to_string(n) + " relations";
            return GPUQO_B200_ERR_CUDA;
        }
        nodes.assign(h_tree, h_tree + nn);
        uint64_t csgs = 0, filt = 0;
        for (int k = 2; k <= n; k++) {
            csgs += h_lvl[k].n_sets;
            filt += binom64(n, k);
            st.fallback_sets += h_lvl[k].n_fb;
        }
        st.connected_sets += csgs;
        st.filtered_subsets += filt;
        st.evaluated_pairs += h_glob->evaluated_pairs;
        st.memo_bytes = (1ull << n) * (sizeof(float4) + 4);
        st.kernel_launches += (uint32_t)n_kernels;
        return 0;
    }

    bool persistent_ok(const std::vector<uint32_t> &blob, DpMode mode) const {
        const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
        return gpuqo_b200_persistent != 0 && !coop_off && !barrier_timed_out && mode == kModeMpdp &&
               h->tree_mode != 0u;
    }

    // stage the blob without building a graph (persistent path)
    int stage(const std::vector<uint32_t> &blob, int n, uint32_t &words, std::string &err) {
        if (int rc = init(err)) return rc;
        words = ((uint32_t)blob.size() + 511u) & ~511u;
        if (int rc = ensure(n, words, err)) return rc;
        std::memset(h_blob, 0, words * 4);
        std::memcpy(h_blob, blob.data(), blob.size() * 4);
        CK(cudaMemcpyAsync(a.blob, h_blob, words * 4, cudaMemcpyHostToDevice, stream));
        return 0;
    }

    int run(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, bool profile,
            std::vector<TreeNode> &nodes, EngineStats &st, std::string &err) {
        if (persistent_ok(blob, mode)) {
            uint32_t pw;
            if (int rc = stage(blob, n, pw, err)) return rc;
            CK(cudaEventRecord(ev0, stream));
            bool launched = false;
            if (int rc = launch_persistent(n, pw, launched, err)) return rc;
            CK(cudaEventRecord(ev1, stream));
            bool failed = true;
            if (launched) {
                if (int rc = barrier_failed(failed, st, err)) return rc;
            }
            if (launched && !failed) {
                if (int rc = finish(n, false, nodes, st, err, true)) return rc;
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, ev0, ev1));
                st.device_ms += ms;
                st.eval_kernel_ms += ms;
                st.eval_kernel_launches += 1;
                return 0;
            }
            // not launched or the barrier timed out: per-level launches below
        }
        uint32_t words;
        cudaGraphExec_t exec;
        if (int rc = prepare(blob, n, mode, ccc, profile, words, exec, err)) return rc;
        CK(cudaEventRecord(ev0, stream));
        if (int rc = launch(exec, err)) return rc;
        CK(cudaEventRecord(ev1, stream));
        if (int rc = finish(n, profile, nodes, st, err)) return rc;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        st.device_ms += ms;
        return 0;
    }

    // Device-resident timing: the planner info is uploaded once, then the DP
    // graph is replayed `iters` times with CUDA events around each replay on
    // the engine's stream; the L2 is flushed (a 256 MB write) between replays
    // outside the timed events.  Returns the mean device ms per replay.
    int time_resident(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, int warmup, int iters,
                      bool flush_l2, double &ms_per_iter, std::vector<TreeNode> &nodes, EngineStats &st,
                      std::string &err) {
        const size_t flush_floats = (256u << 20) / sizeof(float);
        if (persistent_ok(blob, mode)) {
            uint32_t pw;
            if (int rc = stage(blob, n, pw, err)) return rc;
            if (flush_l2 && !flush) CK(cudaMalloc(&flush, flush_floats * sizeof(float)));
            bool usable = true;   // every launch so far started and passed its barriers
            for (int i = 0; i < warmup && usable; i++) {
                bool launched = false, failed = false;
                if (int rc = launch_persistent(n, pw, launched, err)) return rc;
                if (launched)
                    if (int rc = barrier_failed(failed, st, err)) return rc;
                usable = launched && !failed;
            }
            double total = 0.0;
            for (int i = 0; usable && i < iters; i++) {
                if (flush_l2) CK(cudaMemsetAsync(flush, i & 0xFF, flush_floats * sizeof(float), stream));
                bool launched = false, failed = false;
                CK(cudaEventRecord(ev0, stream));
                if (int rc = launch_persistent(n, pw, launched, err)) return rc;
                CK(cudaEventRecord(ev1, stream));
                CK(cudaEventSynchronize(ev1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, ev0, ev1));
                total += ms;
                st.eval_kernel_ms += ms;
                st.eval_kernel_launches += 1;
                if (launched)
                    if (int rc = barrier_failed(failed, st, err)) return rc;
                usable = launched && !failed;
            }
            if (usable && iters > 0) {
                ms_per_iter = total / iters;
                st.device_ms += ms_per_iter;
                return finish(n, false, nodes, st, err, true);
            }
            st.eval_kernel_ms = 0.0;
            st.eval_kernel_launches = 0;
        }
        uint32_t words;
        cudaGraphExec_t exec;
        if (int rc = prepare(blob, n, mode, ccc, false, words, exec, err)) return rc;
        if (flush_l2 && !flush) CK(cudaMalloc(&flush, flush_floats * sizeof(float)));
        for (int i = 0; i < warmup; i++) CK(cudaGraphLaunch(exec, stream));
        double total = 0.0;
        for (int i = 0; i < iters; i++) {
            if (flush_l2) CK(cudaMemsetAsync(flush, i & 0xFF, flush_floats * sizeof(float), stream));
            CK(cudaEventRecord(ev0, stream));
            CK(cudaGraphLaunch(exec, stream));
            CK(cudaEventRecord(ev1, stream));
            CK(cudaEventSynchronize(ev1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ev0, ev1));
            total += ms;
            if (int rc = read_eval_events(n, st, err)) return rc;
        }
        ms_per_iter = iters > 0 ? total / iters : 0.0;
        st.device_ms += ms_per_iter;
        return finish(n, false, nodes, st, err);
    }
};

// One engine of each kind per device, each device's engines and tuning
// record guarded by that device's mutex, so that host threads driving
// different devices (the batch and the server spread over several) do not
// wait for one another.
static std::mutex g_dev_mu[kMaxDevices];
static std::unique_ptr<Engine> g_engines[kMaxDevices];

// the calling thread's current device (a valid index of the engine tables)
static int current_device(int &dev, std::string &err) {
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return GPUQO_B200_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        err = "device index " + std::to_string(dev) + " beyond the library's " + std::to_string(kMaxDevices);
        return GPUQO_B200_ERR_CUDA;
    }
    return 0;
}

}  // namespace gqb

// ===========================================================================
// Entry point that allocates nothing.
//
// Some callers cannot allocate device memory: code that must not leak when
// Postgres aborts a query with elog(ERROR) (a longjmp past any cudaFree),
// processes whose device memory is owned by another pool, and paths with a
// fixed memory budget.  gpuqo_b200_run_noalloc serves them for queries of up
// to kNoAllocMaxRels relations: every scratch buffer of the DP (dense memo,
// level lists, overflow lists, counters, planner-info blob, plan nodes) is
// carved out of the one file-scope array below, which every GPU that loads
// this library holds until the process exits.  Host-side conversion uses
// fixed-size stack buffers; kernels are launched directly on the caller's
// stream (no graph, no events).
//
// In host code g_noalloc_scratch names a host-side stand-in, not the device
// array; its device address comes from cudaGetSymbolAddress, done once per
// device by the first call on that device (so make that first call before
// any stream capture).  All calls share the array: calls that overlap on the
// GPU race with each other.
// ===========================================================================
// Postgres cost GUCs (host_api.cpp / the backend), read the way setParams does
extern "C" double seq_page_cost, cpu_tuple_cost, cpu_operator_cost, disable_cost;
extern "C" int work_mem;
extern "C" bool enable_nestloop, enable_hashjoin;

namespace gqb {

constexpr int kNoAllocMaxRels = 18;
constexpr uint32_t kNoAllocMaxBlobWords = 6144;
constexpr uint64_t kNoAllocMaxSets = 48620;   // C(18, 9), the largest level

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaMemo = 0;
constexpr size_t kNaMemoLeft = kNaMemo + na_align((1ull << kNoAllocMaxRels) * sizeof(float4));
constexpr size_t kNaSets = kNaMemoLeft + na_align((1ull << kNoAllocMaxRels) * sizeof(uint32_t));
constexpr size_t kNaOvfSet = kNaSets + na_align(kNoAllocMaxSets * 4);
constexpr size_t kNaOvfP = kNaOvfSet + na_align(kNoAllocMaxSets * 4);
constexpr size_t kNaOvfOff = kNaOvfP + na_align(kNoAllocMaxSets * 4);
constexpr size_t kNaOvfKey = kNaOvfOff + na_align(kNoAllocMaxSets * 4);
constexpr size_t kNaOvfFirst = kNaOvfKey + na_align(kNoAllocMaxSets * 8);
constexpr size_t kNaLvl = kNaOvfFirst + na_align(kNoAllocMaxSets * 8);
constexpr size_t kNaGlob = kNaLvl + na_align(33 * sizeof(LevelCounters));
constexpr size_t kNaBlob = kNaGlob + na_align(sizeof(GlobalCounters));
constexpr size_t kNaBinom = kNaBlob + na_align(kNoAllocMaxBlobWords * 4);
constexpr size_t kNaTree = kNaBinom + na_align(33 * 33 * 4);
constexpr size_t kNaTreeN = kNaTree + na_align(64 * sizeof(TreeNode));
constexpr size_t kNaTotal = kNaTreeN + na_align(sizeof(int));   // about 6.7 MB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaTotal];

static std::mutex g_na_mu;
static unsigned char *g_na_ptr[64];   // device address of the scratch, per device
static bool g_na_ready[64];

// Once per device, with that device current: resolve the scratch address and
// fill the binomial table.  No allocation.
static int noalloc_setup(int dev) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (g_na_ready[dev]) return 0;
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return GPUQO_B200_ERR_CUDA;
    }
    static uint32_t table[33 * 33];
    for (int i = 0; i <= 32; i++)
        for (int j = 0; j <= 32; j++) {
            uint64_t v = binom64(i, j);
            table[i * 33 + j] = v > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)v;
        }
    e = cudaMemcpy((unsigned char *)ptr + kNaBinom, table, sizeof(table), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: binomial table upload failed: %s\n", cudaGetErrorString(e));
        return GPUQO_B200_ERR_CUDA;
    }
    g_na_ptr[dev] = (unsigned char *)ptr;
    g_na_ready[dev] = true;
    return 0;
}

static inline uint64_t na_bms(const Bitmapset *b) { return (b && b->nwords > 0) ? b->words[0] : 0ull; }
static inline int na_popc(uint64_t x) { return __builtin_popcountll(x); }
static inline uint64_t na_pdep(uint64_t val, uint64_t mask) {
    uint64_t r = 0;
    for (uint64_t bb = 1; mask; bb += bb) {
        uint64_t low = mask & (~mask + 1);
        if (val & bb) r |= low;
        mask &= mask - 1;
    }
    return r;
}
static inline int na_ecidx(int l, int r, int size) {
    if (l > r) { int t = l; l = r; r = t; }
    return l * size - l * (l + 1) / 2 + (r - l - 1);
}

// GpuqoPlannerInfoC -> BFS-relabelled device blob in a caller buffer (the
// same relabelling as bfs_order/relabel/build_blob, in fixed-size storage).
// On failure prints the cause and returns its status code.
static int noalloc_blob(const GpuqoPlannerInfoC *c, uint32_t *blob, uint32_t &words, int *from_of_to) {
    const int n = c->n_rels;
    uint64_t edge[kNoAllocMaxRels];
    for (int i = 0; i < n; i++) {
        if (na_bms(c->base_rels[i].id) != (1ull << (i + 1))) {
            fprintf(stderr, "gpuqo_b200_run_noalloc: base relation %d does not carry relid bit %d\n", i, i + 1);
            return GPUQO_B200_ERR_ARGS;
        }
        edge[i] = na_bms(c->edge_table[i]);
    }
    // BFS order (gpuqo_bfs_indexing.cu:14-55)
    int queue[kNoAllocMaxRels * kNoAllocMaxRels + 1];
    int front = 0, back = 0, nt = 0;
    queue[back++] = 0;
    uint64_t seen = 2ull;
    while (front != back && nt < n) {
        int b = queue[front++];
        from_of_to[nt++] = b;
        uint64_t e = edge[b];
        while (e) {
            int next = __builtin_ffsll((long long)e) - 1;
            if (!(seen & (1ull << next)) && back < kNoAllocMaxRels * kNoAllocMaxRels) queue[back++] = next - 1;
            e &= ~(1ull << next);
        }
        seen |= edge[b];
    }
    if (nt != n) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: the query graph is disconnected\n");
        return GPUQO_B200_ERR_ARGS;
    }
    auto remap = [&](uint64_t m) {
        uint64_t o = 0;
        for (int t = 0; t < n; t++)
            if (m & (1ull << (from_of_to[t] + 1))) o |= 1ull << t;   // compact bit t
        return o;
    };
    int n_ec = 0, n_sels = 0, n_fks = 0;
    for (const EqClassInfo *ec = c->eq_classes; ec; ec = ec->next) {
        int s = na_popc(na_bms(ec->relids));
        n_ec++;
        n_sels += s * (s - 1) / 2;
        n_fks += s;
    }
    words = blob_words_for(n, n_ec, n_sels, n_fks);
    if (n_sels >= 65536 || n_fks >= 65536 || words > kNoAllocMaxBlobWords) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: the planner info needs %u words (%d equivalence classes, %d "
                        "selectivities, %d members); this entry point holds at most %u\n",
                words, n_ec, n_sels, n_fks, kNoAllocMaxBlobWords);
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    for (uint32_t i = 0; i < words; i++) blob[i] = 0u;
    DevHeader *h = reinterpret_cast<DevHeader *>(blob);
    h->n = n;
    h->n_ec = n_ec;
    h->n_sels = n_sels;
    h->n_fks = n_fks;
    h->cpu_operator_cost = (float)cpu_operator_cost;
    h->cpu_tuple_cost = (float)cpu_tuple_cost;
    h->seq_page_cost = (float)seq_page_cost;
    h->disable_cost = (float)disable_cost;
    h->work_mem = work_mem;
    h->enable_nestloop = enable_nestloop ? 1 : 0;
    h->enable_hashjoin = enable_hashjoin ? 1 : 0;
    h->composite_mask = 0;
    h->blob_words = words;
    long long width_sum = 0;
    bool width_ok = true;
    for (int t = 0; t < n; t++) {
        width_sum += c->base_rels[t].width;
        width_ok = width_ok && c->base_rels[t].width >= 0;
    }
    h->hz_packed = (width_ok && width_sum < (1ll << kWidthBits)) ? 1u : 0u;
    for (int t = 0; t < n; t++) {
        const BaseRelationC &b = c->base_rels[from_of_to[t]];
        h->adj[t] = (uint32_t)(remap(edge[from_of_to[t]]) & ~(1ull << t));
        h->rows[t] = b.rows;
        h->tuples[t] = b.tuples;
        h->startup[t] = b.cost.startup;
        h->total[t] = b.cost.total;
        h->width[t] = b.width;
        h->fksel[t] = (float)(1.0 / (double)fmaxf(1.0f, b.tuples));
    }
    DevInfoView v = make_view(blob);
    uint32_t *relids = const_cast<uint32_t *>(v.ec_relids);
    uint32_t *offs = const_cast<uint32_t *>(v.ec_off);
    float *sels = const_cast<float *>(v.sels);
    uint32_t *fks = const_cast<uint32_t *>(v.fks);
    DevVar *vars = const_cast<DevVar *>(v.vars);
    int i = 0, off_sels = 0, off_fks = 0;
    for (const EqClassInfo *ec = c->eq_classes; ec; ec = ec->next, i++) {
        uint64_t ecf = na_bms(ec->relids);     // Postgres bits
        uint64_t ect = remap(ecf);             // compact bits
        int s = na_popc(ecf);
        relids[i] = (uint32_t)ect;
        offs[i] = ((uint32_t)off_sels << 16) | (uint32_t)off_fks;
        for (int lt = 0; lt < s; lt++) {
            uint64_t id_lt = na_pdep(1ull << lt, ect);
            uint64_t id_lf = 1ull << (from_of_to[__builtin_ffsll((long long)id_lt) - 1] + 1);
            int lf = na_popc((id_lf - 1) & ecf);
            for (int rt = lt + 1; rt < s; rt++) {
                uint64_t id_rt = na_pdep(1ull << rt, ect);
                uint64_t id_rf = 1ull << (from_of_to[__builtin_ffsll((long long)id_rt) - 1] + 1);
                int rf = na_popc((id_rf - 1) & ecf);
                sels[off_sels + na_ecidx(lt, rt, s)] = ec->sels[na_ecidx(lf, rf, s)];
            }
            fks[off_fks + lt] = (uint32_t)remap(ec->fk ? na_bms(ec->fk[lf]) : 0ull);
            const VarInfo &vi = ec->vars[lf];
            DevVar &dv = vars[off_fks + lt];
            const int rel_t = __builtin_ffsll((long long)id_lt) - 1;   // compact index of this member
            dv.idx_rows = vi.index.rows;
            dv.idx_startup = vi.index.cost.startup;
            dv.idx_total = vi.index.cost.total;
            dv.flags = (vi.index.available ? 1u : 0u) | (vi.index.unique ? 2u : 0u);
            devvar_bucket_terms(dv, vi.stats.stadistinct, vi.stats.stanullfrac, vi.stats.mcvfreq, h->rows[rel_t],
                                h->tuples[rel_t]);
        }
        off_sels += s * (s - 1) / 2;
        off_fks += s;
    }
    fill_rel_ecs(v, n);
    fill_pair_sel(v);
    return 0;
}

}  // namespace gqb

extern "C" int gpuqo_b200_run_noalloc(int gpuqo_algorithm_arg, const GpuqoPlannerInfoC *info, void *cuda_stream,
                                      GpuqoB200PlanNode *out_nodes, int max_nodes, int *n_nodes) {
    using namespace gqb;
    if (!info || !out_nodes || !n_nodes) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: NULL argument\n");
        return GPUQO_B200_ERR_ARGS;
    }
    const int n = info->n_rels;
    if (n < 1 || n > kNoAllocMaxRels) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: %d relations; this entry point handles 1..%d\n", n,
                kNoAllocMaxRels);
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    if (max_nodes < 2 * n - 1) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: output holds %d nodes, %d needed\n", max_nodes, 2 * n - 1);
        return GPUQO_B200_ERR_ARGS;
    }
    if (gpuqo_spanning_tree_enable) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: plans the query graph as given; gpuqo_spanning_tree_enable is "
                        "served by gpuqo_run\n");
        return GPUQO_B200_ERR_UNSUPPORTED;
    }
    DpMode mode;
    switch (gpuqo_algorithm_arg) {
    case GPUQO_CPU_DPSUB_BICC:
    case GPUQO_CPU_DPSUB_BICC_PARALLEL:
        mode = kModeMpdp;
        break;
    case GPUQO_CPU_DPSUB:
    case GPUQO_CPU_DPSUB_PARALLEL:
    case GPUQO_DPE_DPSUB:
        mode = kModeDpsub;
        break;
    case GPUQO_DPSUB:
        mode = gpuqo_dpsub_bicc_enable ? kModeMpdp : kModeDpsub;
        break;
    default:
        fprintf(stderr, "gpuqo_b200_run_noalloc: algorithm %d is not served by this entry point (DPsub and MPDP "
                        "only)\n", gpuqo_algorithm_arg);
        return GPUQO_B200_ERR_UNSUPPORTED;
    }
    uint32_t blob[kNoAllocMaxBlobWords];
    uint32_t words = 0;
    int from_of_to[kNoAllocMaxRels];
    if (int rc = noalloc_blob(info, blob, words, from_of_to)) return rc;
    // an error left pending by unrelated earlier work would otherwise be
    // reported as this call's own
    cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GPUQO_B200_ERR_CUDA;
    if (int rc = noalloc_setup(dev)) return rc;
    unsigned char *base = g_na_ptr[dev];
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    float4 *memo = (float4 *)(base + kNaMemo);
    uint32_t *memo_left = (uint32_t *)(base + kNaMemoLeft);
    uint32_t *sets = (uint32_t *)(base + kNaSets);
    uint32_t *ovf_set = (uint32_t *)(base + kNaOvfSet);
    uint32_t *ovf_P = (uint32_t *)(base + kNaOvfP);
    uint32_t *ovf_off = (uint32_t *)(base + kNaOvfOff);
    unsigned long long *ovf_key = (unsigned long long *)(base + kNaOvfKey);
    unsigned long long *ovf_first = (unsigned long long *)(base + kNaOvfFirst);
    LevelCounters *lvl = (LevelCounters *)(base + kNaLvl);
    GlobalCounters *glob = (GlobalCounters *)(base + kNaGlob);
    uint32_t *d_blob = (uint32_t *)(base + kNaBlob);
    uint32_t *binom = (uint32_t *)(base + kNaBinom);
    TreeNode *tree = (TreeNode *)(base + kNaTree);
    int *tree_n = (int *)(base + kNaTreeN);
    int sm_count = 148;
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
    const int ccc = gpuqo_dpsub_ccc_enable ? 1 : 0;
    const size_t smem = (size_t)(((words + 3u) & ~3u) + kWarpsPerBlock * kQueueWords) * 4u;

    // every enqueue is checked where it is made, so a failure names its step
    auto failed = [&](cudaError_t e, const char *what) {
        if (e == cudaSuccess) return false;
        fprintf(stderr, "gpuqo_b200_run_noalloc: %s: %s\n", what, cudaGetErrorString(e));
        return true;
    };
    // counters start at zero on every call; the memo needs no clearing (only
    // entries written earlier in the same call are read)
    if (failed(cudaMemcpyAsync(d_blob, blob, words * 4, cudaMemcpyHostToDevice, stream), "planner info upload") ||
        failed(cudaMemsetAsync(lvl, 0, 33 * sizeof(LevelCounters), stream), "counter reset") ||
        failed(cudaMemsetAsync(glob, 0, sizeof(GlobalCounters), stream), "counter reset") ||
        failed(cudaMemsetAsync(tree_n, 0, sizeof(int), stream), "counter reset"))
        return GPUQO_B200_ERR_CUDA;
    k_init_base<<<1, 32, 0, stream>>>(d_blob, memo, memo_left);
    if (failed(cudaGetLastError(), "base relations launch")) return GPUQO_B200_ERR_CUDA;
    for (int k = 2; k <= n; k++) {
        uint64_t total = binom64(n, k);
        uint64_t threads = std::min<uint64_t>((uint64_t)sm_count * 8 * kBlock, (total + 3) / 4);
        threads = std::max<uint64_t>(threads, 32);
        uint32_t per_thread = (uint32_t)((total + threads - 1) / threads);
        uint32_t fblocks = (uint32_t)((total + (uint64_t)per_thread * kBlock - 1) / ((uint64_t)per_thread * kBlock));
        LevelCounters *lc = lvl + k;
        k_filter<<<fblocks, kBlock, 0, stream>>>(d_blob, binom, n, k, total, per_thread, sets, lc);
        int eblocks = (int)std::min<uint64_t>((uint64_t)sm_count * 4, (total + kWarpsPerBlock - 1) / kWarpsPerBlock);
        bool may_overflow = ((1ull << k) - 2ull) > kOvfLimit;
        if (mode == kModeDpsub) {
            k_eval<kModeDpsub><<<eblocks, kBlock, smem, stream>>>(d_blob, words, k, sets, lc, memo, memo_left, ovf_set,
                                                                  ovf_P, ovf_off, ovf_key, ovf_first, glob, ccc);
            if (may_overflow) {
                k_ovf_chunks<kModeDpsub><<<sm_count * 4, kBlock, smem, stream>>>(
                    d_blob, words, k, lc, memo, ovf_set, ovf_P, ovf_off, ovf_key, ovf_first, glob, ccc);
                k_ovf_finalize<kModeDpsub><<<sm_count, kBlock, smem, stream>>>(d_blob, words, lc, memo, memo_left,
                                                                               ovf_set, ovf_key, ovf_first);
            }
        } else {
            k_eval<kModeMpdp><<<eblocks, kBlock, smem, stream>>>(d_blob, words, k, sets, lc, memo, memo_left, ovf_set,
                                                                 ovf_P, ovf_off, ovf_key, ovf_first, glob, ccc);
            if (may_overflow) {
                k_ovf_chunks<kModeMpdp><<<sm_count * 4, kBlock, smem, stream>>>(
                    d_blob, words, k, lc, memo, ovf_set, ovf_P, ovf_off, ovf_key, ovf_first, glob, ccc);
                k_ovf_finalize<kModeMpdp><<<sm_count, kBlock, smem, stream>>>(d_blob, words, lc, memo, memo_left,
                                                                              ovf_set, ovf_key, ovf_first);
            }
        }
        if (failed(cudaGetLastError(), "level launch")) return GPUQO_B200_ERR_CUDA;
    }
    k_extract<<<1, 32, 0, stream>>>(memo, memo_left, (1u << n) - 1u, d_blob, tree, tree_n);
    if (failed(cudaGetLastError(), "plan extraction launch")) return GPUQO_B200_ERR_CUDA;
    TreeNode host_nodes[64];
    int host_n = 0;
    if (failed(cudaMemcpyAsync(host_nodes, tree, 64 * sizeof(TreeNode), cudaMemcpyDeviceToHost, stream),
               "plan download") ||
        failed(cudaMemcpyAsync(&host_n, tree_n, sizeof(int), cudaMemcpyDeviceToHost, stream), "plan download") ||
        failed(cudaStreamSynchronize(stream), "stream synchronisation"))
        return GPUQO_B200_ERR_CUDA;
    if (host_n != 2 * n - 1) {
        fprintf(stderr, "gpuqo_b200_run_noalloc: plan extraction produced %d nodes\n", host_n);
        return GPUQO_B200_ERR_CUDA;
    }
    for (int j = 0; j < host_n; j++) {
        uint64_t orig = 0;
        for (int t = 0; t < n; t++)
            if (host_nodes[j].set & (1u << t)) orig |= 1ull << (from_of_to[t] + 1);
        out_nodes[j].relids = orig;
        out_nodes[j].left = host_nodes[j].left;
        out_nodes[j].right = host_nodes[j].right;
        out_nodes[j].rows = host_nodes[j].rows;
        out_nodes[j].startup = host_nodes[j].startup;
        out_nodes[j].total = host_nodes[j].total;
        out_nodes[j].width = host_nodes[j].width;
    }
    *n_nodes = host_n;
    return GPUQO_B200_OK;
}

// ===========================================================================
// Batched MPDP: many independent queries level by level.  One wave packs the
// memos of its queries into one arena; per level one enumeration launch and
// one evaluation launch serve every query of the wave, so small queries no
// longer pay per-query launch latency.  Items of a level list are
// (query << 32 | set).  The planner info of each query stays in global
// memory (read through the read-only cache) because groups of one warp may
// belong to different queries.
// ===========================================================================
namespace gqb {

struct BatchQ {
    uint32_t blob_off;                 // word offset into the wave's blob buffer
    uint32_t n;
    uint32_t first_base;               // index of its first singleton in the level-1 list
    uint32_t pad;
    unsigned long long memo_off;       // entry offset into the memo arena
    unsigned long long seen_off;       // word offset into the dedup bitmap arena
};

// Sets of a level whose candidate count exceeds kOvfLimit (large biconnected
// blocks: the full set of a cycle, dense sub-graphs), evaluated after the
// level by every warp in chunks of kChunk candidates (kb_dp only).
struct BatchOvf {
    unsigned long long *item;          // [cap] query << 32 | set
    uint32_t *P;                       // [cap] candidate count
    uint32_t *off;                     // [cap] first chunk id (increases with the index)
    unsigned long long *key;           // [cap] min (cost bits << 32 | candidate index) over chunks
    unsigned long long *first;         // [cap] min (first valid candidate << 1 | its cost is NaN)
    uint32_t cap;                      // 0: no overflow list (sets are evaluated by their group)
};

__global__ void kb_init(const BatchQ *__restrict__ qs, int nq, const uint32_t *__restrict__ blobs,
                        float4 *__restrict__ memo, uint32_t *__restrict__ memo_left,
                        unsigned long long *__restrict__ list1, LevelCounters *__restrict__ lvl1) {
    const int q = blockIdx.x;
    if (q >= nq) return;
    const BatchQ Q = qs[q];
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blobs + Q.blob_off);
    for (int i = threadIdx.x; i < (int)Q.n; i += blockDim.x) {
        memo[Q.memo_off + (1ull << i)] =
            base_entry(*h, i);
        memo_left[Q.memo_off + (1ull << i)] = 0u;
        list1[Q.first_base + i] = ((unsigned long long)q << 32) | (1u << i);
    }
    if (threadIdx.x == 0) atomicAdd(&lvl1->n_sets, Q.n);
}

// Warp-aggregated append of 64-bit items to a level list: lanes with ok set
// stage their item in the warp's 64-slot area; every 32 staged items take one
// atomicAdd on the level counter.  Call warp-uniformly; flush with
// stage_flush64 at the end.
__device__ __forceinline__ void stage_emit64(unsigned long long *st, uint32_t &cnt, bool ok,
                                             unsigned long long item, unsigned long long *out, LevelCounters *lc) {
    const int lane = threadIdx.x & 31;
    const uint32_t m = __ballot_sync(kFull, ok);
    if (ok) st[cnt + __popc(m & ((1u << lane) - 1u))] = item;
    cnt += __popc(m);
    __syncwarp();
    if (cnt >= 32) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&lc->n_sets, 32u);
        base = __shfl_sync(kFull, base, 0);
        out[base + lane] = st[lane];
        __syncwarp();
        if (lane < cnt - 32) st[lane] = st[32 + lane];
        cnt -= 32;
        __syncwarp();
    }
}

__device__ __forceinline__ void stage_flush64(unsigned long long *st, uint32_t &cnt, unsigned long long *out,
                                              LevelCounters *lc) {
    const int lane = threadIdx.x & 31;
    if (cnt > 0) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&lc->n_sets, cnt);
        base = __shfl_sync(kFull, base, 0);
        if (lane < cnt) out[base + lane] = st[lane];
    }
    cnt = 0;
    __syncwarp();
}

// connected k-sets of every query, by extension of its (k-1)-sets (c_prev
// items in prev); thread tid of nthreads.  TREE_ONLY (every query of the wave
// tree-shaped): each set is emitted once by the largest-leaf rule of
// level_sets_phase, without the dedup bitmap.
template <bool TREE_ONLY>
__device__ __forceinline__ void batch_extend(const BatchQ *qs, const uint32_t *blobs, const unsigned long long *prev,
                                             uint32_t c_prev, uint32_t *seen, unsigned long long *out,
                                             LevelCounters *lc, unsigned long long *st, uint32_t tid,
                                             uint32_t nthreads) {
    uint32_t cnt = 0;
    const uint32_t rounds = (c_prev + nthreads - 1u) / nthreads;
    for (uint32_t r = 0; r < rounds; r++) {
        const uint32_t idx = tid + r * nthreads;
        uint32_t S = 0u, N = 0u, q = 0u, leaves = 0u;
        unsigned long long seen_off = 0;
        const uint32_t *adj = nullptr;
        if (idx < c_prev) {
            const unsigned long long it = __ldcg(prev + idx);
            q = (uint32_t)(it >> 32);
            S = (uint32_t)it;
            const BatchQ Q = qs[q];
            adj = reinterpret_cast<const DevHeader *>(blobs + Q.blob_off)->adj;
            seen_off = Q.seen_off;
            uint32_t x = S;
            while (x) {
                int v = __ffs(x) - 1;
                x &= x - 1u;
                const uint32_t a = __ldg(adj + v);
                N |= a;
                if (TREE_ONLY && __popc(a & S) == 1) leaves |= 1u << v;
            }
            N &= ~S;
        }
        const bool single = (S & (S - 1u)) == 0u;
        const int deg = __popc(N);
        const int maxdeg = (int)__reduce_max_sync(kFull, (uint32_t)deg);
        for (int j = 0; j < maxdeg; j++) {
            bool ok = false;
            unsigned long long item = 0;
            if (j < deg) {
                const uint32_t bitv = N & (0u - N);
                N ^= bitv;
                const uint32_t T = S | bitv;
                if (TREE_ONLY) {
                    const uint32_t p = __ldg(adj + (__ffs(bitv) - 1)) & S;   // v's only neighbour in S
                    ok = (single ? S : (leaves & ~p)) < bitv;                // v is T's largest leaf
                } else {
                    const uint32_t bm = 1u << (T & 31u);
                    ok = !(atomicOr(&seen[seen_off + (T >> 5)], bm) & bm);
                }
                item = ((unsigned long long)q << 32) | T;
            }
            stage_emit64(st, cnt, ok, item, out, lc);
        }
    }
    stage_flush64(st, cnt, out, lc);
}

__global__ void __launch_bounds__(kBlock) kb_level_sets(const BatchQ *__restrict__ qs,
                                                        const uint32_t *__restrict__ blobs,
                                                        const unsigned long long *__restrict__ prev,
                                                        const LevelCounters *__restrict__ prev_lc,
                                                        uint32_t *__restrict__ seen,
                                                        unsigned long long *__restrict__ out,
                                                        LevelCounters *__restrict__ lc) {
    __shared__ unsigned long long stage[kWarpsPerBlock][64];
    const int warp = threadIdx.x >> 5;
    batch_extend<false>(qs, blobs, prev, __ldcg(&prev_lc->n_sets), seen, out, lc, stage[warp],
                 blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// candidate c of a tree-shaped query (see k_eval_tree): edge {a, b}, a < b
__device__ __forceinline__ void tree_cand(const DevHeader &h, uint32_t S, int a, int b, uint32_t c, uint32_t &L,
                                          uint32_t &R, uint32_t &p, uint32_t &ecm, bool masked) {
    const uint32_t *tab = reinterpret_cast<const uint32_t *>(&h) + h.tree_tab;
    const int n = h.n, nn = n * n;
    const int rt = __ffs(S) - 1;
    const uint32_t *anc_r = tab + 2 * nn + rt * n;
    const int ch = ((__ldg(anc_r + b) >> a) & 1u) ? b : a;
    const uint32_t comp_c = S & __ldg(tab + rt * n + ch);
    const uint32_t comp_a = (ch == a) ? comp_c : (S ^ comp_c);
    const uint32_t side = c & 1u;
    L = side ? (S ^ comp_a) : comp_a;
    R = S ^ L;
    const uint32_t post =
        (uint32_t)(__popc(S & __ldg(tab + nn + rt * n + ch)) - __popc(S & __ldg(anc_r + ch)) + __popc(comp_c) - 1);
    p = h.index_order ? dpsub_index(L, S) : 2u * post + side;
    ecm = 0u;
    if (masked) {
        const int ch0 = ((__ldg(tab + 2 * nn + b) >> a) & 1u) ? b : a;
        ecm = h.edge_ec[ch0];
    }
}

// ALL_MASKED (with TREE_ONLY): every query of the wave has only two-member
// classes on tree edges (DevHeader::ec_masked), so the general class pass
// is not compiled in
template <int G, bool TREE_ONLY, bool ALL_MASKED = false>
__device__ __forceinline__ void batch_groups(const BatchQ *qs, const uint32_t *blobs, uint32_t first, uint32_t stride,
                                             const unsigned long long *items, uint32_t count, int k, float4 *memo_all,
                                             uint32_t *memo_left_all, unsigned long long &pairs,
                                             const BatchOvf &ovf, LevelCounters *lc) {
    const int lane = threadIdx.x & 31;
    const int grp = lane / G, gl = lane % G;
    const uint32_t group_mask = (G == 32) ? kFull : (((1u << G) - 1u) << (grp * G));
    Blocks B;
    CycleCache cc;
    for (uint32_t base = first; base < count; base += stride) {
        const uint32_t i = base + (uint32_t)grp;
        const bool has = i < count;
        unsigned long long it = has ? __ldcg(items + i) : 0ull;
        const uint32_t q = (uint32_t)(it >> 32), S = (uint32_t)it;
        BatchQ Q;
        Q.blob_off = 0;
        Q.memo_off = 0;
        if (has) Q = qs[q];
        const DevInfoView d = make_view(blobs + Q.blob_off);
        const DevHeader &h = *d.h;
        float4 *memo = memo_all + Q.memo_off;
        uint32_t *memo_left = memo_left_all + Q.memo_off;
        const bool tree = has && (TREE_ONLY || h.tree_mode != 0u);
        const bool masked = ALL_MASKED || (tree && h.ec_masked != 0u);
        uint32_t P = 0;
        B.nb = 0;
        if (has) {
            if (tree) {
                P = 2u * (uint32_t)(k - 1);
            } else if (!TREE_ONLY) {
                find_blocks(S, h.adj, B);
                P = B.etotal;
                if (ovf.cap != 0u && P > kOvfLimit) {
                    // to the level's overflow list; one packed atomic assigns the
                    // list index and the first chunk id in the same order
                    if (gl == 0) {
                        const uint32_t nch = (P + kChunk - 1u) / kChunk;
                        const unsigned long long old = atomicAdd(&lc->ovf_packed, (1ull << 40) | nch);
                        const uint32_t idx = (uint32_t)(old >> 40);
                        if (idx < ovf.cap) {
                            ovf.item[idx] = it;
                            ovf.P[idx] = P;
                            ovf.off[idx] = (uint32_t)(old & 0xFFFFFFFFFFull);
                            ovf.key[idx] = ~0ull;
                            ovf.first[idx] = ~0ull;
                        }
                    }
                    P = 0u;   // no candidate here, no memo write
                }
            }
        }
        __syncwarp();
        const uint32_t iters = __reduce_max_sync(kFull, (P + G - 1u) / G);
        LaneBest best;
        best.init();
        EdgeIter ei;
        ei.vs = S;
        ei.nb = 0u;
        ei.v = 0;
        ei.e = 0u;
        int ea = 0, eb = 0, bcur = 0;
        for (uint32_t j = 0; j < iters; j++) {
            const uint32_t c = (uint32_t)gl + j * G;
            const bool active = has && c < P;
            uint32_t L = 0, R = 0, p = 0, ecm = 0;
            bool valid = false;
            if (active) {
                if (tree) {
                    while (ei.e <= (c >> 1)) edge_next(h.adj, S, ei, ea, eb);
                    tree_cand(h, S, ea, eb, c, L, R, p, ecm, masked);
                    valid = true;
                } else if (!TREE_ONLY) {
                    uint32_t key;
                    valid = mpdp_candidate(S, B, h.adj, c, bcur, L, R, key, cc);
                    p = valid ? key_index(h, key, L, S) : key;
                }
            }
            if (valid) {
                RelVal l = load_rel(memo, L, d.h->hz_packed), r = load_rel(memo, R, d.h->hz_packed);
                RelVal out = (ALL_MASKED || masked) ? join_eval_t<true>(d, L, l, R, r, ecm)
                                                    : join_eval_t<false>(d, L, l, R, r, 0u);
                best_update(best, p, L, out);
            }
        }
        uint32_t kh = (uint32_t)(best.key >> 32), kl = (uint32_t)best.key, fp = best.first_p;
#pragma unroll
        for (int off = G / 2; off >= 1; off >>= 1) {
            uint32_t oh = __shfl_xor_sync(kFull, kh, off);
            uint32_t ol = __shfl_xor_sync(kFull, kl, off);
            uint32_t of = __shfl_xor_sync(kFull, fp, off);
            if (oh < kh || (oh == kh && ol < kl)) {
                kh = oh;
                kl = ol;
            }
            if (of < fp) fp = of;
        }
        const bool nan_first = has && best.first_p == fp && best.first_nan;
        const unsigned nm = __ballot_sync(kFull, nan_first) & group_mask;
        const unsigned long long gkey = ((unsigned long long)kh << 32) | kl;
        if (has) {
            if (nm) {
                if (nan_first) memo_write(*d.h, memo, memo_left, S, best.nan_val, best.nan_left);
            } else if (best.key == gkey && best.key != ~0ull) {
                memo_write(*d.h, memo, memo_left, S, best.val, best.left);
            }
        }
        pairs += best.n_valid;
    }
}

__global__ void __launch_bounds__(kBlock) kb_eval(const BatchQ *__restrict__ qs, const uint32_t *__restrict__ blobs,
                                                  const unsigned long long *__restrict__ items,
                                                  const LevelCounters *__restrict__ lc, int k,
                                                  float4 *__restrict__ memo, uint32_t *__restrict__ memo_left,
                                                  GlobalCounters *__restrict__ glob, uint32_t target_lanes,
                                                  int max_group) {
    const uint32_t count = __ldcg(&lc->n_sets);
    if (count == 0u) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int G = 2;
    while (G < max_group && (uint64_t)count * (uint64_t)G < (uint64_t)target_lanes) G <<= 1;
    G = G <= 2 ? 2 : (G <= 8 ? 8 : 32);
    const uint32_t gwarp = blockIdx.x * kWarpsPerBlock + warp;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    unsigned long long pairs = 0;
    BatchOvf none;
    none.cap = 0u;
    LevelCounters *lcw = nullptr;
    if (G == 2) batch_groups<2, false>(qs, blobs, gwarp * 16, nwarps * 16, items, count, k, memo, memo_left, pairs, none, lcw);
    else if (G == 8) batch_groups<8, false>(qs, blobs, gwarp * 4, nwarps * 4, items, count, k, memo, memo_left, pairs, none, lcw);
    else batch_groups<32, false>(qs, blobs, gwarp, nwarps, items, count, k, memo, memo_left, pairs, none, lcw);
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

// Overflow chunks of level lc: every warp takes chunks of kChunk candidates
// of a listed set (eval_range with the CCC queue) and folds its winner into
// the set's keys with 64-bit atomicMin, as k_ovf_chunks does for one query.
__device__ __forceinline__ void batch_ovf_chunks(const BatchQ *qs, const uint32_t *blobs, LevelCounters *lc,
                                                 const float4 *memo_all, const BatchOvf &ovf, uint32_t *queue,
                                                 unsigned long long &pairs) {
    const int lane = threadIdx.x & 31;
    const unsigned long long packed = __ldcg(&lc->ovf_packed);
    const uint32_t n_ovf = (uint32_t)(packed >> 40);
    const uint32_t n_chunks = (uint32_t)(packed & 0xFFFFFFFFFFull);
    Blocks B;
    B.nb = 0;
    uint32_t cur_idx = kFull;
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(&lc->chunk_next, 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= n_chunks) break;
        uint32_t lo_i = 0, hi_i = n_ovf - 1u;   // largest idx with off[idx] <= c
        while (lo_i < hi_i) {
            const uint32_t mid = (lo_i + hi_i + 1u) >> 1;
            if (__ldcg(ovf.off + mid) <= c) lo_i = mid;
            else hi_i = mid - 1u;
        }
        const uint32_t idx = lo_i;
        const unsigned long long it = __ldcg(ovf.item + idx);
        const uint32_t q = (uint32_t)(it >> 32), S = (uint32_t)it;
        const uint32_t P = __ldcg(ovf.P + idx);
        const BatchQ Q = qs[q];
        const DevInfoView d = make_view(blobs + Q.blob_off);
        if (idx != cur_idx) find_blocks(S, d.h->adj, B);
        cur_idx = idx;
        const uint32_t lo = (c - __ldcg(ovf.off + idx)) * kChunk;
        const uint32_t hi = lo + kChunk < P ? lo + kChunk : P;
        LaneBest best;
        best.init();
        eval_range<kModeMpdp>(d, d.h->adj, S, B, lo, hi, memo_all + Q.memo_off, queue, true, best);
        unsigned long long mk, fk;
        warp_winner(best, mk, fk);
        if (lane == 0) {
            if (mk != ~0ull) atomicMin(ovf.key + idx, mk);
            atomicMin(ovf.first + idx, fk);
        }
        pairs += best.n_valid;
    }
}

// Winner of every listed set: the candidate the keys name is evaluated again
// and written to the memo (k_ovf_finalize for one query).
__device__ __forceinline__ void batch_ovf_finalize(const BatchQ *qs, const uint32_t *blobs, LevelCounters *lc,
                                                   float4 *memo_all, uint32_t *memo_left_all, const BatchOvf &ovf,
                                                   uint32_t tid, uint32_t nthreads) {
    const uint32_t n_ovf = (uint32_t)(__ldcg(&lc->ovf_packed) >> 40);
    for (uint32_t idx = tid; idx < n_ovf; idx += nthreads) {
        const unsigned long long it = __ldcg(ovf.item + idx);
        const uint32_t q = (uint32_t)(it >> 32), S = (uint32_t)it;
        const BatchQ Q = qs[q];
        const DevInfoView d = make_view(blobs + Q.blob_off);
        const uint32_t *adj = d.h->adj;
        float4 *memo = memo_all + Q.memo_off;
        const unsigned long long first = __ldcg(ovf.first + idx);
        const uint32_t p = (first & 1ull) ? (uint32_t)(first >> 1) : (uint32_t)__ldcg(ovf.key + idx);
        uint32_t L, R;
        if (d.h->index_order) {   // plain-DPsub index
            L = pdep32(p + 1u, S);
            R = S ^ L;
        } else {
            Blocks B;
            find_blocks(S, adj, B);
            int b = 0;
            while (b + 1 < B.nb && B.prefix[b + 1] <= p) b++;
            const uint32_t blk = B.mask[b];
            const uint32_t lb = pdep32(p - B.prefix[b] + 1u, blk);
            const uint32_t rb = blk ^ lb;
            L = grow(lowest(lb), S & ~rb, adj);
            R = grow(lowest(rb), S & ~lb, adj);
        }
        const RelVal l = load_rel(memo, L, d.h->hz_packed), r = load_rel(memo, R, d.h->hz_packed);
        const RelVal out = join_eval(d, L, l, R, r);
        memo_write(*d.h, memo, memo_left_all + Q.memo_off, S, out, L);
    }
}

__global__ void kb_extract(const BatchQ *__restrict__ qs, int nq, const uint32_t *__restrict__ blobs,
                           const float4 *__restrict__ memo, const uint32_t *__restrict__ memo_left,
                           TreeNode *__restrict__ out, int *__restrict__ n_out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const BatchQ Q = qs[q];
    const uint32_t wmask =
        reinterpret_cast<const DevHeader *>(blobs + Q.blob_off)->hz_packed ? kWidthMask : 0xFFFFFFFFu;
    const uint32_t full = (Q.n == 32) ? 0xFFFFFFFFu : ((1u << Q.n) - 1u);
    TreeNode *o = out + (size_t)q * 64;
    const float4 *m = memo + Q.memo_off;
    const uint32_t *ml = memo_left + Q.memo_off;
    int n = 0;
    uint32_t stack_set[64];
    int stack_parent[64], stack_side[64];
    int sp = 0;
    stack_set[sp] = full;
    stack_parent[sp] = -1;
    stack_side[sp] = 0;
    sp++;
    while (sp > 0 && n < 64) {
        sp--;
        uint32_t s = stack_set[sp];
        int parent = stack_parent[sp], side = stack_side[sp];
        float4 v = __ldcg(m + s);
        TreeNode t;
        t.set = s;
        t.left = -1;
        t.right = -1;
        t.rows = v.x;
        t.startup = v.y;
        t.total = v.z;
        t.width = (int)(__float_as_uint(v.w) & wmask);
        int me = n++;
        o[me] = t;
        if (parent >= 0) {
            if (side == 0) o[parent].left = me;
            else o[parent].right = me;
        }
        uint32_t l = __ldcg(ml + s) & s;
        if (__popc(s) > 1 && l != 0u && l != s && sp + 2 <= 64) {
            stack_set[sp] = s ^ l;
            stack_parent[sp] = me;
            stack_side[sp] = 1;
            sp++;
            stack_set[sp] = l;
            stack_parent[sp] = me;
            stack_side[sp] = 0;
            sp++;
        }
    }
    n_out[q] = n;
}

// kb_dp: a whole wave of queries in ONE cooperative, persistent launch.
// Phase 0 writes every query's base relations and emits its level-2 sets
// (one warp per query, one lane per relation: each edge once, from its lower
// end).  Then, per level k, the grid evaluates level k of every query while
// it enumerates level k+1, with a grid barrier between levels; the plans are
// extracted (one thread per query) after the last level.  The grid barrier
// is bounded (grid_barrier); on timeout the host reruns the wave with
// per-level launches.
template <bool TREE_ONLY, bool ALL_MASKED = false>
__global__ void __launch_bounds__(kBlock, TREE_ONLY ? 3 : 2) kb_dp(const BatchQ *__restrict__ qs, int nq, int maxn,
                                                   const uint32_t *__restrict__ blobs, float4 *__restrict__ memo,
                                                   uint32_t *__restrict__ memo_left, uint32_t *__restrict__ seen,
                                                   unsigned long long *__restrict__ listA,
                                                   unsigned long long *__restrict__ listB,
                                                   LevelCounters *__restrict__ lvl, GlobalCounters *__restrict__ glob,
                                                   TreeNode *__restrict__ tree, int *__restrict__ tree_n,
                                                   unsigned *__restrict__ bar, uint32_t target_lanes,
                                                   BatchOvf ovf, unsigned poll_limit) {
    const unsigned max_polls = barrier_polls(poll_limit);
    __shared__ unsigned long long stage[kWarpsPerBlock][64];
    __shared__ uint32_t queues[kWarpsPerBlock][kQueueWords];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long *st = stage[warp];
    const uint32_t gwarp = blockIdx.x * kWarpsPerBlock + warp;
    const uint32_t nwarps = gridDim.x * kWarpsPerBlock;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nthreads = gridDim.x * blockDim.x;
    unsigned long long pairs = 0;
    unsigned epoch = 0;   // grid barriers passed (thread 0)

    // phase 0 (gpuqo_cpu_sequential.cu:80-92 for the base entries)
    {
        uint32_t cnt = 0;
        for (uint32_t q = gwarp; q < (uint32_t)nq; q += nwarps) {
            const BatchQ Q = qs[q];
            const DevHeader *h = reinterpret_cast<const DevHeader *>(blobs + Q.blob_off);
            const int v = lane;
            uint32_t nb = 0u;
            if (v < (int)Q.n) {
                memo[Q.memo_off + (1ull << v)] = base_entry(*h, v);
                memo_left[Q.memo_off + (1ull << v)] = 0u;
                nb = __ldg(h->adj + v) & ~((2u << v) - 1u);
            }
            const int deg = __popc(nb);
            const int maxdeg = (int)__reduce_max_sync(kFull, (uint32_t)deg);
            for (int j = 0; j < maxdeg; j++) {
                const bool ok = j < deg;
                unsigned long long item = 0;
                if (ok) {
                    const int u = __ffs(nb) - 1;
                    nb &= nb - 1u;
                    item = ((unsigned long long)q << 32) | (1u << v) | (1u << u);
                }
                stage_emit64(st, cnt, ok, item, listA, lvl + 2);
            }
        }
        stage_flush64(st, cnt, listA, lvl + 2);
    }
    if (!grid_barrier<false>(bar, epoch, max_polls)) return;

    for (int k = 2; k <= maxn; k++) {
        unsigned long long *cur = (k & 1) ? listB : listA;
        unsigned long long *nxt = (k & 1) ? listA : listB;
        const uint32_t count = __ldcg(&lvl[k].n_sets);
        // enumeration from the far end of the grid, evaluation from the start
        if (k < maxn) batch_extend<TREE_ONLY>(qs, blobs, cur, count, seen, nxt, lvl + k + 1, st, nthreads - 1u - tid, nthreads);
        int max_group = 1;
        while (max_group < 32 && max_group < 2 * (k - 1)) max_group <<= 1;
        int G = 2;
        while (G < max_group && (uint64_t)count * (uint64_t)G < (uint64_t)target_lanes) G <<= 1;
        G = G <= 2 ? 2 : (G <= 8 ? 8 : 32);
        LevelCounters *lk = lvl + k;
        if (G == 2)
            batch_groups<2, TREE_ONLY, ALL_MASKED>(qs, blobs, gwarp * 16, nwarps * 16, cur, count, k, memo, memo_left,
                                                   pairs, ovf, lk);
        else if (G == 8)
            batch_groups<8, TREE_ONLY, ALL_MASKED>(qs, blobs, gwarp * 4, nwarps * 4, cur, count, k, memo, memo_left,
                                                   pairs, ovf, lk);
        else
            batch_groups<32, TREE_ONLY, ALL_MASKED>(qs, blobs, gwarp, nwarps, cur, count, k, memo, memo_left, pairs,
                                                    ovf, lk);
        if (!grid_barrier<false>(bar, epoch, max_polls)) return;
        if (TREE_ONLY) continue;   // tree sets have 2(k - 1) candidates: never an overflow
        // overflow sets of level k: the counter is final after the barrier, so
        // every block takes the same branch.  A list longer than its capacity
        // is left to the host (the affected queries are rerun one by one).
        const uint32_t n_ovf = (uint32_t)(__ldcg(&lk->ovf_packed) >> 40);
        if (n_ovf != 0u && n_ovf <= ovf.cap) {
            batch_ovf_chunks(qs, blobs, lk, memo, ovf, queues[warp], pairs);
            if (!grid_barrier<false>(bar, epoch, max_polls)) return;
            batch_ovf_finalize(qs, blobs, lk, memo, memo_left, ovf, tid, nthreads);
            if (!grid_barrier<false>(bar, epoch, max_polls)) return;
        }
    }

    for (uint32_t q = tid; q < (uint32_t)nq; q += nthreads) {
        const BatchQ Q = qs[q];
        const uint32_t full = (Q.n == 32) ? 0xFFFFFFFFu : ((1u << Q.n) - 1u);
        const uint32_t wmask =
            reinterpret_cast<const DevHeader *>(blobs + Q.blob_off)->hz_packed ? kWidthMask : 0xFFFFFFFFu;
        extract_plan(memo + Q.memo_off, memo_left + Q.memo_off, full, wmask, tree + (size_t)q * 64, tree_n + q);
    }
    pairs = __reduce_add_sync(kFull, (uint32_t)pairs);
    if (lane == 0 && pairs) atomicAdd(&glob->evaluated_pairs, pairs);
}

// Candidate bound of a query for the batch (the batch has no overflow path):
// sum over blocks of 2^|b| - 2 with |b| <= the graph's largest block.
static uint64_t mpdp_candidate_bound(int n, int max_block) {
    int bmax = std::min(std::max(max_block, 2), std::max(n, 2));
    uint64_t nblk = (uint64_t)(n - 1 + bmax - 2) / (uint64_t)(bmax - 1);
    return nblk * ((1ull << bmax) - 2ull);
}

bool batch_eligible(const std::vector<uint32_t> &blob) {
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
    return h->n >= 1 && h->n <= 30;
}

// true when some set of the query may have more candidates than one group
// evaluates: those sets need the overflow phase of kb_dp
static bool batch_needs_ovf(const std::vector<uint32_t> &blob) {
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
    return mpdp_candidate_bound(h->n, (int)h->max_block) > kOvfLimit;
}

constexpr uint64_t kBatchOvfCap = 1ull << 22;   // overflow list entries per wave (32 B each)

// Connected sets of a tree-shaped query graph (its connected subtrees): with
// f(v) = prod over children c of (1 + f(c)) for the tree rooted at relation
// 0, the count is the sum of f(v).  Exact, O(n).
static double tree_connected_sets(const DevHeader *h) {
    const int n = h->n;
    int order[32], parent[32], m = 0;
    uint32_t seen = 1u;
    order[m++] = 0;
    parent[0] = -1;
    for (int i = 0; i < m; i++) {
        uint32_t nb = h->adj[order[i]] & ~seen;
        seen |= nb;
        while (nb) {
            const int c = __builtin_ctz(nb);
            nb &= nb - 1u;
            parent[c] = order[i];
            order[m++] = c;
        }
    }
    double f[32], total = 0.0;
    for (int i = 0; i < n; i++) f[i] = 1.0;
    for (int i = m - 1; i >= 0; i--) {
        const int v = order[i];
        total += f[v];
        if (parent[v] >= 0) f[parent[v]] *= 1.0 + f[v];
    }
    return total;
}

// A tree-shaped query with this many connected sets fills the GPU on its own:
// the single-query kernel (k_dp_tree, planner info in shared memory) then
// evaluates more pairs per second than a batch wave, so the batch hands it over.
// (Tuning::batch_single_sets, 2^20 until the autotuner measures it)
static bool batch_prefers_single(const std::vector<uint32_t> &blob, int device) {
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
    return h->tree_mode != 0u && gpuqo_b200_persistent != 0 &&
           tree_connected_sets(h) > g_tuning[device].batch_single_sets;
}

double engine_work_estimate(const std::vector<uint32_t> &blob) {
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
    const double n = (double)h->n;
    if (h->tree_mode) return tree_connected_sets(h) * 2.0 * std::max(n - 1.0, 1.0);
    return std::ldexp(1.0, h->n) * n;
}

uint64_t batch_query_bytes(int n) {
    const uint64_t slots = 1ull << n;
    return slots * (sizeof(float4) + 4) + slots / 8 + 2 * max_level_sets(n) * 8 + 64 * sizeof(TreeNode) + 4096;
}

struct BatchEngine {
    int device = -1, sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // arena (grown on demand)
    uint64_t cap_slots = 0, cap_items = 0, cap_words = 0, cap_seen = 0;
    int cap_q = 0;
    float4 *memo = nullptr;
    uint32_t *memo_left = nullptr, *blobs = nullptr, *seen = nullptr;
    unsigned long long *listA = nullptr, *listB = nullptr;
    BatchQ *qs = nullptr;
    TreeNode *tree = nullptr;
    int *tree_n = nullptr;
    LevelCounters *lvl = nullptr;
    GlobalCounters *glob = nullptr;
    unsigned *bar = nullptr, *h_bar = nullptr;   // grid barrier words of kb_dp (device, pinned copy)
    int coop_grid = -1;                          // co-resident blocks of kb_dp<false> (0: no cooperative launch)
    int coop_grid_tree = -1;                     // co-resident blocks of kb_dp<true>
    int coop_grid_masked = -1;                   // co-resident blocks of kb_dp<true, true>
    bool barrier_timed_out = false;              // a grid barrier of kb_dp gave up: per-level launches until reset
    BatchOvf ovf{};                              // overflow list of kb_dp
    uint64_t cap_ovf = 0;
    void *flush = nullptr;                       // L2 flush buffer (device-resident timing only)
    // pinned staging of a wave: planner infos and descriptors in, plans and
    // counters out (grown on demand; the copies are truly asynchronous)
    unsigned char *h_in = nullptr, *h_out = nullptr;
    size_t cap_h_in = 0, cap_h_out = 0;

    static int grow_pinned(unsigned char *&p, size_t &cap, size_t bytes, std::string &err) {
        if (bytes <= cap) return 0;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        CK(cudaMallocHost(&p, bytes));
        cap = bytes;
        return 0;
    }

    int init(std::string &err) {
        if (stream) return 0;
        CK(cudaGetDevice(&device));
        CK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
        CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&ev0));
        CK(cudaEventCreate(&ev1));
        CK(cudaMalloc(&lvl, 33 * sizeof(LevelCounters)));
        CK(cudaMalloc(&glob, sizeof(GlobalCounters)));
        CK(cudaMalloc(&bar, 4 * sizeof(unsigned)));
        CK(cudaMallocHost(&h_bar, 4 * sizeof(unsigned)));
        int dev_coop = 0, occ = 0, occ_tree = 0, occ_masked = 0;
        cudaDeviceGetAttribute(&dev_coop, cudaDevAttrCooperativeLaunch, device);
        coop_grid = coop_grid_tree = coop_grid_masked = 0;
        if (dev_coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kb_dp<false>, kBlock, 0) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_tree, kb_dp<true>, kBlock, 0) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_masked, kb_dp<true, true>, kBlock, 0) == cudaSuccess) {
            coop_grid = occ * sm_count;
            coop_grid_tree = occ_tree * sm_count;
            coop_grid_masked = occ_masked * sm_count;
        }
        cudaGetLastError();
        return 0;
    }

    // per-level launches of one wave (the queries, blobs and arena are staged)
    uint32_t enqueue_levels(int nq, int maxn, uint64_t seen_words) {
        cudaMemsetAsync(lvl, 0, 33 * sizeof(LevelCounters), stream);
        cudaMemsetAsync(glob, 0, sizeof(GlobalCounters), stream);
        cudaMemsetAsync(seen, 0, seen_words * 4, stream);
        kb_init<<<nq, 32, 0, stream>>>(qs, nq, blobs, memo, memo_left, listA, lvl + 1);
        uint32_t kernels = 1;
        const uint32_t target_lanes = (uint32_t)sm_count * 24u * 32u;
        for (int k = 2; k <= maxn; k++) {
            unsigned long long *prev = (k & 1) ? listB : listA;
            unsigned long long *cur = (k & 1) ? listA : listB;
            kb_level_sets<<<sm_count * 8, kBlock, 0, stream>>>(qs, blobs, prev, lvl + (k - 1), seen, cur, lvl + k);
            int max_group = 1;
            while (max_group < 32 && max_group < 2 * (k - 1)) max_group <<= 1;
            kb_eval<<<sm_count * 4, kBlock, 0, stream>>>(qs, blobs, cur, lvl + k, k, memo, memo_left, glob,
                                                         target_lanes, max_group);
            kernels += 2;
        }
        kb_extract<<<(nq + 127) / 128, 128, 0, stream>>>(qs, nq, blobs, memo, memo_left, tree, tree_n);
        return kernels + 1;
    }

    // the wave as one cooperative launch of kb_dp (kb_dp<true> when every query
    // is tree-shaped, kb_dp<true, true> when every class of every query is also
    // a two-member class on a tree edge); false when it could not start
    bool enqueue_persistent(int nq, int maxn, uint64_t seen_words, bool tree_only, bool all_masked) {
        const bool masked = tree_only && all_masked;
        const int grid = masked ? coop_grid_masked : (tree_only ? coop_grid_tree : coop_grid);
        if (grid <= 0 || gpuqo_b200_persistent == 0 || barrier_timed_out) return false;
        cudaMemsetAsync(lvl, 0, 33 * sizeof(LevelCounters), stream);
        cudaMemsetAsync(glob, 0, sizeof(GlobalCounters), stream);
        if (!tree_only) cudaMemsetAsync(seen, 0, seen_words * 4, stream);
        cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), stream);
        uint32_t target_lanes = (uint32_t)grid * kBlock;
        unsigned poll_limit = (unsigned)std::max(0, gpuqo_b200_barrier_poll_limit);
        void *args[] = {&qs, &nq, &maxn, &blobs, &memo, &memo_left, &seen, &listA, &listB,
                        &lvl, &glob, &tree, &tree_n, &bar, &target_lanes, &ovf, &poll_limit};
        const void *fn = masked ? (const void *)kb_dp<true, true>
                                : (tree_only ? (const void *)kb_dp<true> : (const void *)kb_dp<false>);
        if (cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), args, 0, stream) != cudaSuccess) {
            cudaGetLastError();
            coop_grid = coop_grid_tree = coop_grid_masked = 0;
            return false;
        }
        return true;
    }

    // grows geometrically (twice the old capacity when that is more than the
    // need) so that waves of changing composition do not reallocate the arena
    // every time; falls back to the exact need when the larger block does
    // not fit
    template <class T> int grow(T *&p, uint64_t &cap, uint64_t need, std::string &err) {
        if (need <= cap) return 0;
        if (p) cudaFree(p);
        p = nullptr;
        const uint64_t want = std::max(need, 2 * cap);
        cap = 0;
        if (want > need && cudaMalloc(&p, want * sizeof(T)) == cudaSuccess) {
            cap = want;
            return 0;
        }
        cudaGetLastError();
        p = nullptr;
        CK(cudaMalloc(&p, need * sizeof(T)));
        cap = need;
        return 0;
    }

    bool persistent_ready() const {
        return coop_grid > 0 && coop_grid_tree > 0 && gpuqo_b200_persistent != 0 && !barrier_timed_out;
    }

    // One wave: all queries' memos fit.  wb: per query planner-info blob.
    // Queries that this wave could not finish (sets beyond the group limit
    // without the overflow phase, or an overfull overflow list) are listed in
    // redo (wave-local indices) for the single-query engine.
    int run_wave(const std::vector<const std::vector<uint32_t> *> &wb, std::vector<std::vector<TreeNode>> &out,
                 std::vector<int> &redo, EngineStats &st, double &ms, std::string &err) {
        redo.clear();
        std::vector<int> need_ovf;
        for (int q = 0; q < (int)wb.size(); q++)
            if (batch_needs_ovf(*wb[q])) need_ovf.push_back(q);
        if (!need_ovf.empty() && !persistent_ready()) {
            // per-level launches cannot split a set: those queries run alone
            std::vector<const std::vector<uint32_t> *> rest;
            std::vector<int> idx;
            size_t j = 0;
            for (int q = 0; q < (int)wb.size(); q++) {
                if (j < need_ovf.size() && need_ovf[j] == q) {
                    j++;
                    continue;
                }
                rest.push_back(wb[q]);
                idx.push_back(q);
            }
            out.assign(wb.size(), {});
            redo = need_ovf;
            ms = 0.0;
            if (rest.empty()) return 0;
            std::vector<std::vector<TreeNode>> rout;
            bool ovf_full = false;
            if (int rc = stage_and_run(rest, rout, st, ms, ovf_full, err)) return rc;
            for (size_t i = 0; i < idx.size(); i++) out[idx[i]] = std::move(rout[i]);
            return 0;
        }
        bool ovf_full = false;
        if (int rc = stage_and_run(wb, out, st, ms, ovf_full, err)) return rc;
        if (ovf_full) redo = need_ovf;
        return 0;
    }

    int stage_and_run(const std::vector<const std::vector<uint32_t> *> &wb, std::vector<std::vector<TreeNode>> &out,
                      EngineStats &st, double &ms, bool &ovf_full, std::string &err) {
        const int nq = (int)wb.size();
        std::vector<BatchQ> hq(nq);
        uint64_t slots = 0, words = 0, seen_words = 0, items = 0, base = 0, ovf_need = 0;
        int maxn = 0;
        bool tree_only = true, all_masked = true;
        for (int q = 0; q < nq; q++) {
            const DevHeader *h = reinterpret_cast<const DevHeader *>(wb[q]->data());
            const int n = h->n;
            hq[q].blob_off = (uint32_t)words;
            hq[q].n = (uint32_t)n;
            hq[q].first_base = (uint32_t)base;
            hq[q].memo_off = slots;
            hq[q].seen_off = seen_words;
            words += (wb[q]->size() + 3) & ~(size_t)3;
            slots += 1ull << n;
            seen_words += std::max<uint64_t>((1ull << n) / 32, 1);
            items += max_level_sets(n);
            base += (uint64_t)n;
            maxn = std::max(maxn, n);
            if (batch_needs_ovf(*wb[q])) ovf_need += max_level_sets(n);
            tree_only = tree_only && h->tree_mode != 0u;
            all_masked = all_masked && h->ec_masked != 0u;
        }
        items = std::max(items, base);
        ovf_need = std::min(ovf_need, kBatchOvfCap);
        if (int rc = over_budget(slots * (sizeof(float4) + 4) + words * 4 + seen_words * 4 + items * 16 + ovf_need * 32,
                                 "the batch wave's arena", err))
            return rc;
        uint64_t c1 = cap_slots, c2 = cap_slots, c3 = cap_words, c4 = cap_seen, c5 = cap_items, c6 = cap_items;
        if (int rc = grow(memo, c1, slots, err)) return rc;
        if (int rc = grow(memo_left, c2, slots, err)) return rc;
        cap_slots = std::min(c1, c2);
        if (int rc = grow(blobs, c3, words, err)) return rc;
        cap_words = c3;
        if (int rc = grow(seen, c4, seen_words, err)) return rc;
        cap_seen = c4;
        if (int rc = grow(listA, c5, items, err)) return rc;
        if (int rc = grow(listB, c6, items, err)) return rc;
        cap_items = std::min(c5, c6);
        if (ovf_need > cap_ovf) {
            uint64_t a1 = cap_ovf, a2 = cap_ovf, a3 = cap_ovf, a4 = cap_ovf, a5 = cap_ovf;
            if (int rc = grow(ovf.item, a1, ovf_need, err)) return rc;
            if (int rc = grow(ovf.P, a2, ovf_need, err)) return rc;
            if (int rc = grow(ovf.off, a3, ovf_need, err)) return rc;
            if (int rc = grow(ovf.key, a4, ovf_need, err)) return rc;
            if (int rc = grow(ovf.first, a5, ovf_need, err)) return rc;
            cap_ovf = ovf_need;
        }
        ovf.cap = (uint32_t)ovf_need;
        if (nq > cap_q) {
            cudaFree(qs);
            cudaFree(tree);
            cudaFree(tree_n);
            qs = nullptr;
            tree = nullptr;
            tree_n = nullptr;
            cap_q = 0;
            CK(cudaMalloc(&qs, nq * sizeof(BatchQ)));
            CK(cudaMalloc(&tree, (size_t)nq * 64 * sizeof(TreeNode)));
            CK(cudaMalloc(&tree_n, nq * sizeof(int)));
            cap_q = nq;
        }
        // stage the planner infos and the descriptors in pinned memory (the
        // previous wave's copies ended with its synchronisation)
        const size_t in_blob = (size_t)words * 4, in_q = (size_t)nq * sizeof(BatchQ);
        if (int rc = grow_pinned(h_in, cap_h_in, in_blob + in_q, err)) return rc;
        uint32_t *hblob = reinterpret_cast<uint32_t *>(h_in);
        for (int q = 0; q < nq; q++) {
            const size_t len = wb[q]->size(), padded = (len + 3) & ~(size_t)3;
            std::memcpy(hblob + hq[q].blob_off, wb[q]->data(), len * 4);
            std::memset(hblob + hq[q].blob_off + len, 0, (padded - len) * 4);
        }
        std::memcpy(h_in + in_blob, hq.data(), in_q);
        CK(cudaMemcpyAsync(blobs, hblob, in_blob, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(qs, h_in + in_blob, in_q, cudaMemcpyHostToDevice, stream));
        // plans and counters come back into pinned memory, with the barrier
        // words, in one synchronisation
        const size_t o_tree = 0, o_n = o_tree + (size_t)nq * 64 * sizeof(TreeNode),
                     o_lvl = (o_n + (size_t)nq * sizeof(int) + 15) & ~(size_t)15,
                     o_glob = o_lvl + 33 * sizeof(LevelCounters), o_end = o_glob + sizeof(GlobalCounters);
        if (int rc = grow_pinned(h_out, cap_h_out, o_end, err)) return rc;
        auto download = [&]() -> int {
            CK(cudaMemcpyAsync(h_out + o_tree, tree, (size_t)nq * 64 * sizeof(TreeNode), cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(h_out + o_n, tree_n, nq * sizeof(int), cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(h_out + o_lvl, lvl, 33 * sizeof(LevelCounters), cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(h_out + o_glob, glob, sizeof(GlobalCounters), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            CK(cudaGetLastError());
            return 0;
        };
        uint32_t kernels = 1;
        CK(cudaEventRecord(ev0, stream));
        bool persistent = enqueue_persistent(nq, maxn, seen_words, tree_only, all_masked);
        CK(cudaGetLastError());
        if (persistent) CK(cudaMemcpyAsync(h_bar, bar, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        if (!persistent) {
            ovf.cap = 0u;
            kernels = enqueue_levels(nq, maxn, seen_words);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev1, stream));
        if (int rc = download()) return rc;
        if (persistent && h_bar[2] != 0u) {   // barrier timed out: rerun with per-level launches
            persistent = false;
            barrier_timed_out = true;           // and use them until gpuqo_b200_reset_persistent
            st.barrier_timeouts++;
            CK(cudaEventRecord(ev0, stream));
            ovf.cap = 0u;
            kernels = enqueue_levels(nq, maxn, seen_words);
            CK(cudaGetLastError());
            CK(cudaEventRecord(ev1, stream));
            if (int rc = download()) return rc;
        }
        const TreeNode *htree = reinterpret_cast<const TreeNode *>(h_out + o_tree);
        const int *hn = reinterpret_cast<const int *>(h_out + o_n);
        const LevelCounters *hl = reinterpret_cast<const LevelCounters *>(h_out + o_lvl);
        const GlobalCounters &hg = *reinterpret_cast<const GlobalCounters *>(h_out + o_glob);
        float fms = 0.f;
        CK(cudaEventElapsedTime(&fms, ev0, ev1));
        ms = fms;
        // kb_dp skipped the overflow phase of a level whose list outgrew its
        // capacity; the per-level launches (ovf.cap 0) evaluate every set in
        // its group and need no redo
        ovf_full = false;
        for (int k = 2; k <= maxn; k++)
            if (persistent && (uint32_t)(hl[k].ovf_packed >> 40) > ovf.cap) ovf_full = true;
        out.resize(nq);
        for (int q = 0; q < nq; q++) {
            if (hn[q] != 2 * (int)hq[q].n - 1 && !(ovf_full && batch_needs_ovf(*wb[q]))) {
                err = "batched plan extraction produced " + std::to_string(hn[q]) + " nodes";
                return GPUQO_B200_ERR_CUDA;
            }
            out[q].assign(htree + (size_t)q * 64, htree + (size_t)q * 64 + std::max(hn[q], 0));
        }
        for (int k = 2; k <= maxn; k++) st.connected_sets += hl[k].n_sets;
        st.evaluated_pairs += hg.evaluated_pairs;
        st.memo_bytes = std::max<uint64_t>(st.memo_bytes, slots * (sizeof(float4) + 4));
        st.device_ms += fms;
        st.kernel_launches += kernels;
        return 0;
    }
};

static std::unique_ptr<BatchEngine> g_batch[kMaxDevices];

int engine_run_batch(const std::vector<const std::vector<uint32_t> *> &blobs, uint64_t wave_bytes,
                     std::vector<std::vector<TreeNode>> &out, EngineStats &st, std::vector<double> &wave_ms,
                     std::string &err) {
    int dev = 0;
    if (int rc = current_device(dev, err)) return rc;
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    auto &be = g_batch[dev];
    if (!be) be.reset(new BatchEngine());
    if (int rc = be->init(err)) return rc;
    out.assign(blobs.size(), {});
    auto &eng = g_engines[dev];
    // large tree-shaped queries: one persistent single-query launch each
    std::vector<size_t> rest;
    for (size_t i = 0; i < blobs.size(); i++) {
        if (!batch_prefers_single(*blobs[i], dev)) {
            rest.push_back(i);
            continue;
        }
        if (!eng) eng.reset(new Engine());
        const int n = reinterpret_cast<const DevHeader *>(blobs[i]->data())->n;
        const double before = st.device_ms;
        if (int rc = eng->run(*blobs[i], n, kModeMpdp, true, false, out[i], st, err)) return rc;
        st.handoff_ms += st.device_ms - before;
    }
    // tree-shaped queries first (waves of kb_dp<true>), then the others; the
    // order within each part is the caller's (largest first)
    std::stable_partition(rest.begin(), rest.end(), [&](size_t i) {
        return reinterpret_cast<const DevHeader *>(blobs[i]->data())->tree_mode != 0u;
    });
    // waves: consecutive queries while the wave's memory stays within budget
    // and its queries are all tree-shaped or all not
    size_t r = 0;
    while (r < rest.size()) {
        std::vector<const std::vector<uint32_t> *> wave;
        std::vector<size_t> idx;
        uint64_t bytes = 0;
        const bool wave_tree = reinterpret_cast<const DevHeader *>(blobs[rest[r]]->data())->tree_mode != 0u;
        while (r < rest.size()) {
            const size_t i = rest[r];
            const DevHeader *hi = reinterpret_cast<const DevHeader *>(blobs[i]->data());
            const int n = hi->n;
            const uint64_t b = batch_query_bytes(n);
            if (!wave.empty() && (bytes + b > wave_bytes || (hi->tree_mode != 0u) != wave_tree)) break;
            wave.push_back(blobs[i]);
            idx.push_back(i);
            bytes += b;
            r++;
        }
        std::vector<std::vector<TreeNode>> wout;
        std::vector<int> redo;
        double ms = 0;
        if (int rc = be->run_wave(wave, wout, redo, st, ms, err)) return rc;
        wave_ms.push_back(ms);
        for (size_t j = 0; j < idx.size(); j++) out[idx[j]] = std::move(wout[j]);
        if (!redo.empty()) {
            if (!eng) eng.reset(new Engine());
            for (int r : redo) {
                const std::vector<uint32_t> &b = *wave[r];
                const int n = reinterpret_cast<const DevHeader *>(b.data())->n;
                std::vector<TreeNode> nodes;
                if (int rc = eng->run(b, n, kModeMpdp, true, false, nodes, st, err)) return rc;
                out[idx[r]] = std::move(nodes);
            }
        }
    }
    return 0;
}


// One exact DP.  Tree-shaped graphs run k_dp_tree (Engine); other graphs
// under MPDP enumeration (MPDP, and plain DPsub on valid pairs) run as a
// one-query wave of the general persistent kernel kb_dp<false>, which has the
// overflow phases in the same launch; the per-level launches of Engine serve
// the rest (plain all-subsets DPsub, no cooperative launch, an overfull
// overflow list, gpuqo_b200_persistent = 0).
int engine_run(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, bool profile,
               std::vector<TreeNode> &nodes, EngineStats &stats, std::string &err) {
    if (n < 1 || n > 31) {
        err = "exact DP supports 1..31 relations";
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    int dev = 0;
    if (int rc = current_device(dev, err)) return rc;
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
    if (mode == kModeMpdp && h->tree_mode == 0u && n <= 30 && gpuqo_b200_persistent != 0 && !profile) {
        auto &be = g_batch[dev];
        if (!be) be.reset(new BatchEngine());
        if (int rc = be->init(err)) return rc;
        if (be->persistent_ready()) {
            std::vector<const std::vector<uint32_t> *> wave(1, &blob);
            std::vector<std::vector<TreeNode>> wout;
            std::vector<int> redo;
            EngineStats st;
            double ms = 0.0;
            if (int rc = be->run_wave(wave, wout, redo, st, ms, err)) return rc;
            if (redo.empty()) {
                nodes = std::move(wout[0]);
                stats.connected_sets += st.connected_sets;
                stats.filtered_subsets += st.filtered_subsets;
                stats.evaluated_pairs += st.evaluated_pairs;
                stats.memo_bytes = st.memo_bytes;
                stats.device_ms += st.device_ms;
                stats.kernel_launches += st.kernel_launches;
                stats.barrier_timeouts += st.barrier_timeouts;
                return 0;
            }
        }
    }
    auto &eng = g_engines[dev];
    if (!eng) eng.reset(new Engine());
    return eng->run(blob, n, mode, ccc, profile, nodes, stats, err);
}

int engine_time_resident(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, int warmup, int iters,
                         bool flush_l2, double &ms_per_iter, std::vector<TreeNode> &nodes, EngineStats &stats,
                         std::string &err) {
    if (n < 1 || n > 31) {
        err = "exact DP supports 1..31 relations";
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    int dev = 0;
    if (int rc = current_device(dev, err)) return rc;
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    // the same routing as engine_run: graphs with cycles as one-query waves
    const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
    if (mode == kModeMpdp && h->tree_mode == 0u && n <= 30 && gpuqo_b200_persistent != 0 && iters > 0) {
        auto &be = g_batch[dev];
        if (!be) be.reset(new BatchEngine());
        if (int rc = be->init(err)) return rc;
        if (be->persistent_ready()) {
            std::vector<const std::vector<uint32_t> *> wave(1, &blob);
            const size_t flush_bytes = 256u << 20;
            if (flush_l2 && !be->flush) CK(cudaMalloc(&be->flush, flush_bytes));
            double total = 0.0;
            bool ok = true;
            for (int i = 0; ok && i < warmup + iters; i++) {
                if (flush_l2) CK(cudaMemsetAsync(be->flush, i & 0xFF, flush_bytes, be->stream));
                std::vector<std::vector<TreeNode>> wout;
                std::vector<int> redo;
                EngineStats st;
                double ms = 0.0;
                if (int rc = be->run_wave(wave, wout, redo, st, ms, err)) return rc;
                ok = redo.empty();
                if (i >= warmup) total += ms;
                if (ok && i == warmup + iters - 1) {
                    nodes = std::move(wout[0]);
                    stats.connected_sets += st.connected_sets;
                    stats.filtered_subsets += st.filtered_subsets;
                    stats.evaluated_pairs += st.evaluated_pairs;
                    stats.memo_bytes = st.memo_bytes;
                    stats.kernel_launches += st.kernel_launches;
                }
                stats.barrier_timeouts += st.barrier_timeouts;
            }
            if (ok) {
                ms_per_iter = total / iters;
                stats.device_ms += ms_per_iter;
                return 0;
            }
        }
    }
    auto &eng = g_engines[dev];
    if (!eng) eng.reset(new Engine());
    return eng->time_resident(blob, n, mode, ccc, warmup, iters, flush_l2, ms_per_iter, nodes, stats, err);
}

// ---------------------------------------------------------------------------
// Autotuner.  On tree-shaped blobs of growing size (the host passes synthetic
// stars) it times k_dp_tree<2>, <3> and <4> device-resident, and one batch
// wave holding about 2^24 connected sets against single launches, then
// installs in the device's tuning record the three crossovers: up to which
// count of connected sets per level the 2-blocks variant beats the 3-blocks
// one at that size and every smaller one, from which count per level the
// 4-blocks variant wins at that size and every larger one (per level: the
// variants trade latency against throughput within a level, and the count per
// level carries over from stars to deeper trees, where the total does not),
// and from which total count a single launch beats its share of a wave.
// ---------------------------------------------------------------------------
static double crossover(const std::vector<double> &sets, const std::vector<bool> &wins) {
    size_t i = wins.size();
    while (i > 0 && wins[i - 1]) i--;
    if (i == wins.size()) return 1e30;     // never wins
    if (i == 0) return 0.0;                // wins from the smallest size on
    return std::sqrt(sets[i - 1] * sets[i]);
}

// the same from below: the largest count up to which `wins` holds at every size
static double crossover_below(const std::vector<double> &sets, const std::vector<bool> &wins) {
    size_t i = 0;
    while (i < wins.size() && wins[i]) i++;
    if (i == 0) return 0.0;                // loses at the smallest size
    if (i == wins.size()) return 1e30;     // wins at every size
    return std::sqrt(sets[i - 1] * sets[i]);
}

int engine_autotune(const std::vector<std::vector<uint32_t>> &blobs, double &single_narrow_level_sets,
                    double &single_wide_level_sets, double &batch_single_sets, std::string &err) {
    int dev = 0;
    if (int rc = current_device(dev, err)) return rc;
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    auto &eng = g_engines[dev];
    if (!eng) eng.reset(new Engine());
    auto &be = g_batch[dev];
    if (!be) be.reset(new BatchEngine());
    if (int rc = be->init(err)) return rc;
    std::vector<double> sets, level_sets;
    std::vector<bool> narrow_wins, wide_wins, single_wins;
    for (const auto &blob : blobs) {
        const DevHeader *h = reinterpret_cast<const DevHeader *>(blob.data());
        if (!h->tree_mode) continue;
        double t[3] = {0.0, 0.0, 0.0};   // k_dp_tree<2>, <3>, <4>
        for (int v = 0; v < 3; v++) {
            eng->force_minb = 2 + v;
            std::vector<TreeNode> nodes;
            EngineStats st;
            const int rc = eng->time_resident(blob, h->n, kModeMpdp, true, 1, 3, false, t[v], nodes, st, err);
            eng->force_minb = 0;
            if (rc) return rc;
        }
        const double cs = tree_connected_sets(h);
        const int m = (int)std::min(256.0, std::max(2.0, std::ceil(double(1u << 24) / cs)));
        std::vector<const std::vector<uint32_t> *> wave(m, &blob);
        double wms = 0.0;
        for (int rep = 0; rep < 2; rep++) {   // the first wave sizes the arena
            std::vector<std::vector<TreeNode>> wout;
            std::vector<int> redo;
            EngineStats st;
            if (int rc = be->run_wave(wave, wout, redo, st, wms, err)) return rc;
        }
        sets.push_back(cs);
        level_sets.push_back(cs / h->n);
        // each variant against the best of the other two, so that the
        // crossovers give the fastest of the three at every measured size
        narrow_wins.push_back(t[0] < std::min(t[1], t[2]));
        wide_wins.push_back(t[2] < std::min(t[0], t[1]));
        single_wins.push_back(std::min(t[0], std::min(t[1], t[2])) < wms / m);
    }
    single_narrow_level_sets = crossover_below(level_sets, narrow_wins);
    single_wide_level_sets = crossover(level_sets, wide_wins);
    batch_single_sets = crossover(sets, single_wins);
    Tuning &tu = g_tuning[dev];
    tu.single_narrow_level_sets = single_narrow_level_sets;
    tu.single_wide_level_sets = single_wide_level_sets;
    tu.batch_single_sets = batch_single_sets;
    tu.tuned = true;
    return 0;
}

void engine_set_tuning(double single_narrow_level_sets, double single_wide_level_sets, double batch_single_sets,
                       bool tuned) {
    int dev = 0;
    std::string err;
    if (current_device(dev, err)) dev = 0;   // no device yet: the record of device 0
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    Tuning &tu = g_tuning[dev];
    tu.single_narrow_level_sets = single_narrow_level_sets;
    tu.single_wide_level_sets = single_wide_level_sets;
    tu.batch_single_sets = batch_single_sets;
    tu.tuned = tuned;
}

int engine_reset_persistent() {
    int dev = 0;
    std::string err;
    if (current_device(dev, err)) return 0;
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    int cleared = 0;
    if (g_engines[dev] && g_engines[dev]->barrier_timed_out) {
        g_engines[dev]->barrier_timed_out = false;
        cleared++;
    }
    if (g_batch[dev] && g_batch[dev]->barrier_timed_out) {
        g_batch[dev]->barrier_timed_out = false;
        cleared++;
    }
    return cleared;
}

void engine_get_tuning(double &single_narrow_level_sets, double &single_wide_level_sets, double &batch_single_sets, bool &tuned) {
    int dev = 0;
    std::string err;
    if (current_device(dev, err)) dev = 0;
    std::lock_guard<std::mutex> lk(g_dev_mu[dev]);
    const Tuning &tu = g_tuning[dev];
    single_narrow_level_sets = tu.single_narrow_level_sets;
    single_wide_level_sets = tu.single_wide_level_sets;
    batch_single_sets = tu.batch_single_sets;
    tuned = tu.tuned;
}

}  // namespace gqb
