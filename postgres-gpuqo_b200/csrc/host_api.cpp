// host_api.cpp - C ABI of libgpuqo_b200.so: gpuqo_run, the GUC variables,
// conversion of the planner's C structures, BFS relabelling, plan output.
//
// The flow of one call mirrors __gpuqo_run (gpuqo_main_internal.cu:82-160):
// convert -> BFS relabel -> exact DP (or IDP driver) -> map the plan back ->
// palloc'd QueryTreeC.  The exact DP runs on the GPU (dp_kernels.cu).
#include <algorithm>
#include <cmath>
#include <csignal>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "dp_engine.h"
#include "gpuqo_b200.h"
#include "host_idp.h"
#include "host_info.h"

// ---------------------------------------------------------------------------
// Postgres backend symbols.  Weak: inside postgres the backend's own
// definitions win; standalone (tests, bench) these stand in.
// ---------------------------------------------------------------------------
extern "C" {
__attribute__((weak)) void *palloc(size_t size) { return malloc(size ? size : 1); }
__attribute__((weak)) void *palloc0(size_t size) { return calloc(1, size ? size : 1); }
__attribute__((weak)) void pfree(void *p) { free(p); }
__attribute__((weak)) volatile sig_atomic_t InterruptPending = 0;
__attribute__((weak)) void ProcessInterrupts(void) {}

// Postgres cost GUCs read by setParams (gpuqo_planner_info.cu:84-131),
// with Postgres defaults and the enable_* settings the reference's cost model
// assumes (README "Limitations").
__attribute__((weak)) double seq_page_cost = 1.0;
__attribute__((weak)) double random_page_cost = 4.0;
__attribute__((weak)) double cpu_tuple_cost = 0.01;
__attribute__((weak)) double cpu_index_tuple_cost = 0.005;
__attribute__((weak)) double cpu_operator_cost = 0.0025;
__attribute__((weak)) int effective_cache_size = 524288;
__attribute__((weak)) double disable_cost = 1.0e10;
__attribute__((weak)) bool enable_seqscan = true;
__attribute__((weak)) bool enable_indexscan = true;
__attribute__((weak)) bool enable_tidscan = false;
__attribute__((weak)) bool enable_sort = true;
__attribute__((weak)) bool enable_hashagg = true;
__attribute__((weak)) bool enable_nestloop = true;
__attribute__((weak)) bool enable_mergejoin = false;
__attribute__((weak)) bool enable_hashjoin = true;
__attribute__((weak)) int work_mem = 4096;

// gpuqo GUC variables, initialised to the boot values of guc.c
// (src/backend/utils/misc/guc.c:1103-1170, 2140-2297, 4810-4826).
__attribute__((weak)) int gpuqo_algorithm = GPUQO_DPSIZE;   // defined by gpuqo_main.c in postgres
int gpuqo_scratchpad_size_mb = 10;
int gpuqo_max_memo_size_mb = 1024;
int gpuqo_min_memo_size_mb = 1;
int gpuqo_n_parallel = 10240;
bool gpuqo_dpsub_filter_enable = true;
int gpuqo_dpsub_filter_threshold = 16;
int gpuqo_dpsub_filter_cpu_enum_threshold = 1024;
int gpuqo_dpsub_filter_keys_overprovisioning = 100;
bool gpuqo_dpsub_ccc_enable = true;
bool gpuqo_dpsub_csg_enable = true;
int gpuqo_dpsub_csg_threshold = 128;
bool gpuqo_dpsub_tree_enable = false;
bool gpuqo_dpsub_bicc_enable = false;
int gpuqo_dpe_n_threads = 4;
int gpuqo_dpe_pairs_per_depbuf = 128;
int gpuqo_cpu_dpsub_parallel_chunk_size = 64;
bool gpuqo_spanning_tree_enable = false;
int gpuqo_idp_n_iters = 0;
int gpuqo_idp_type = GPUQO_IDP2;
int gpuqo_dplin_csg_threshold_lindp = 10000;
int gpuqo_dplin_threshold_lindp = 14;
int gpuqo_dplin_threshold_idp = 100;

int gpuqo_b200_profile_kernels = 0;
int gpuqo_b200_batch_memory_mb = 32768;
int gpuqo_b200_persistent = 1;
int gpuqo_b200_barrier_poll_limit = 0;
int gpuqo_b200_device_memory_mb = 0;
int gpuqo_b200_devices = 1;
int gpuqo_b200_sparse_from_rels = 32;
int gpuqo_b200_sparse_host_list = 0;
int gpuqo_b200_server_batch_window_us = 100;
}

namespace gqb {

static thread_local int t_last_error = GPUQO_B200_OK;
static thread_local GpuqoB200Stats t_stats;

void set_error(int code, const std::string &msg) {
    t_last_error = code;
    if (code != GPUQO_B200_OK) fprintf(stderr, "gpuqo_b200: %s\n", msg.c_str());
}

void stats_reset() { memset(&t_stats, 0, sizeof(t_stats)); }

void stats_add(const EngineStats &s) {
    t_stats.connected_sets += s.connected_sets;
    t_stats.evaluated_pairs += s.evaluated_pairs;
    t_stats.filtered_subsets += s.filtered_subsets;
    if (s.memo_bytes > t_stats.memo_bytes) t_stats.memo_bytes = s.memo_bytes;
    t_stats.device_ms += s.device_ms;
    t_stats.eval_kernel_ms += s.eval_kernel_ms;
    t_stats.eval_kernel_launches += s.eval_kernel_launches;
    t_stats.kernel_launches += s.kernel_launches;
    t_stats.fallback_sets += s.fallback_sets;
    t_stats.barrier_timeouts += s.barrier_timeouts;
    t_stats.handoff_device_ms += s.handoff_ms;
    t_stats.n_subproblems += 1;
}

static inline int popc64(mask64 x) { return __builtin_popcountll(x); }
static inline mask64 lowest64(mask64 x) { return x & (~x + 1); }
static inline int lowest_pos64(mask64 x) { return __builtin_ffsll((long long)x) - 1; }
static inline mask64 bit64(int n) { return (mask64)1 << n; }
static inline mask64 pdep64(mask64 val, mask64 mask) {
    mask64 r = 0;
    for (mask64 bb = 1; mask; bb += bb) {
        mask64 low = lowest64(mask);
        if (val & bb) r |= low;
        mask &= mask - 1;
    }
    return r;
}
static inline int ec_nsels(int s) { return s * (s - 1) / 2; }
static inline int ec_index(int l, int r, int size) {
    if (l > r) std::swap(l, r);
    return l * size - l * (l + 1) / 2 + (r - l - 1);
}

HostParams read_params() {
    HostParams p;
    p.effective_cache_size = (float)effective_cache_size;
    p.random_page_cost = (float)random_page_cost;
    p.seq_page_cost = (float)seq_page_cost;
    p.cpu_tuple_cost = (float)cpu_tuple_cost;
    p.cpu_index_tuple_cost = (float)cpu_index_tuple_cost;
    p.cpu_operator_cost = (float)cpu_operator_cost;
    p.disable_cost = (float)disable_cost;
    p.enable_seqscan = enable_seqscan;
    p.enable_indexscan = enable_indexscan;
    p.enable_tidscan = enable_tidscan;
    p.enable_sort = enable_sort;
    p.enable_hashagg = enable_hashagg;
    p.enable_nestloop = enable_nestloop;
    p.enable_mergejoin = enable_mergejoin;
    p.enable_hashjoin = enable_hashjoin;
    p.work_mem = work_mem;
    return p;
}

static mask64 bms_word0(const Bitmapset *b, bool &wide) {
    if (!b) return 0;
    for (int i = 1; i < b->nwords; i++)
        if (b->words[i]) wide = true;
    return b->nwords > 0 ? b->words[0] : 0;
}

bool convert_info(const GpuqoPlannerInfoC *c, HostInfo &out, std::string &err) {
    if (!c || c->n_rels < 1) {
        err = "empty planner info";
        return false;
    }
    if (c->n_rels >= 64) {
        err = "64-bit conversion called with >= 64 relations";
        return false;
    }
    bool wide = false;
    out.n = c->n_rels;
    out.p = read_params();
    out.base.resize(out.n);
    out.edge.resize(out.n);
    for (int i = 0; i < out.n; i++) {
        out.edge[i] = bms_word0(c->edge_table[i], wide);
        HostBaseRel &b = out.base[i];
        b.id = bms_word0(c->base_rels[i].id, wide);
        b.rows = c->base_rels[i].rows;
        b.tuples = c->base_rels[i].tuples;
        b.width = c->base_rels[i].width;
        b.cost = c->base_rels[i].cost;
        b.composite = false;
        if (b.id != bit64(i + 1)) {
            err = "base relation " + std::to_string(i) + " does not carry relid bit " + std::to_string(i + 1);
            return false;
        }
    }
    out.ec_relids.clear();
    out.ec_sels.clear();
    out.ec_fks.clear();
    out.ec_vars.clear();
    for (const EqClassInfo *ec = c->eq_classes; ec != NULL; ec = ec->next) {
        mask64 r = bms_word0(ec->relids, wide);
        out.ec_relids.push_back(r);
        int s = popc64(r);
        for (int j = 0; j < ec_nsels(s); j++) out.ec_sels.push_back(ec->sels[j]);
        for (int j = 0; j < s; j++) {
            out.ec_fks.push_back(ec->fk ? bms_word0(ec->fk[j], wide) : 0);
            out.ec_vars.push_back(ec->vars[j]);
        }
    }
    if (wide) {
        err = "relation ids beyond the 64-bit range";
        return false;
    }
    return true;
}

std::vector<int> bfs_order(const HostInfo &info) {
    std::vector<int> order;
    std::vector<int> queue;
    queue.reserve(info.n);
    queue.push_back(0);
    size_t front = 0;
    mask64 seen = bit64(1);
    while (front < queue.size() && (int)order.size() < info.n) {
        int b = queue[front++];
        mask64 edges = info.edge[b];
        order.push_back(b);
        while (edges) {
            int next = lowest_pos64(edges);
            if (!(seen & bit64(next))) queue.push_back(next - 1);
            edges &= ~bit64(next);
        }
        seen |= info.edge[b];
    }
    return order;
}

HostInfo relabel(const HostInfo &from, const std::vector<int> &from_of_to) {
    const int nt = (int)from_of_to.size();
    std::vector<int> to_of_from(64, -1);
    for (int t = 0; t < nt; t++) to_of_from[from_of_to[t]] = t;
    // bit f + 1 (relation f) -> bit to_of_from[f] + 1; bits of relations
    // outside from_of_to (and bit 0) are dropped
    auto remap = [&](mask64 m) {
        mask64 o = 0;
        for (m &= ~1ull; m; m &= m - 1) {
            const int t = to_of_from[__builtin_ctzll(m) - 1];
            if (t >= 0) o |= bit64(t + 1);
        }
        return o;
    };
    HostInfo to;
    to.n = nt;
    to.p = from.p;
    to.base.resize(nt);
    to.edge.resize(nt);
    for (int t = 0; t < nt; t++) {
        to.edge[t] = remap(from.edge[from_of_to[t]]) & ~bit64(t + 1);
        to.base[t] = from.base[from_of_to[t]];
        to.base[t].id = bit64(t + 1);
    }
    to.ec_relids.resize(from.ec_relids.size());
    to.ec_sels.resize(from.ec_sels.size());
    to.ec_fks.resize(from.ec_fks.size());
    to.ec_vars.resize(from.ec_vars.size());
    int off_sels = 0, off_fks = 0;
    for (size_t i = 0; i < from.ec_relids.size(); i++) {
        mask64 ecf = from.ec_relids[i];
        mask64 ect = remap(ecf);
        int s = popc64(ecf);
        to.ec_relids[i] = ect;
        for (int lt = 0; lt < s; lt++) {
            mask64 id_lt = pdep64(bit64(lt), ect);
            mask64 id_lf = bit64(from_of_to[lowest_pos64(id_lt) - 1] + 1);
            int lf = popc64((lowest64(id_lf) - 1) & ecf);
            for (int rt = lt + 1; rt < s; rt++) {
                mask64 id_rt = pdep64(bit64(rt), ect);
                mask64 id_rf = bit64(from_of_to[lowest_pos64(id_rt) - 1] + 1);
                int rf = popc64((lowest64(id_rf) - 1) & ecf);
                to.ec_sels[off_sels + ec_index(lt, rt, s)] = from.ec_sels[off_sels + ec_index(lf, rf, s)];
            }
            to.ec_fks[off_fks + lt] = remap(from.ec_fks[off_fks + lf]);
            to.ec_vars[off_fks + lt] = from.ec_vars[off_fks + lf];
        }
        off_sels += ec_nsels(s);
        off_fks += s;
    }
    return to;
}

// Size of the largest biconnected block of the query graph (Hopcroft-Tarjan
// over compact adjacency masks).  Every block of a connected subset lies
// inside a block of the whole graph, so this bounds the MPDP candidate count
// of every set: sum over blocks of 2^|b| - 2 with sum(|b| - 1) = |S| - 1.
static int max_block_size(const HostInfo &info) {
    const int n = info.n;
    if (n <= 1) return n;
    std::vector<uint32_t> adj(n);
    for (int i = 0; i < n; i++) adj[i] = (uint32_t)(info.edge[i] >> 1);
    std::vector<int> disc(n, -1), low(n, 0), parent(n, -1), vstk, stk_u;
    std::vector<uint32_t> stk_e;
    int t = 0, best = 1;
    for (int root = 0; root < n; root++) {
        if (disc[root] >= 0) continue;
        disc[root] = low[root] = t++;
        vstk.push_back(root);
        stk_u.push_back(root);
        stk_e.push_back(adj[root]);
        while (!stk_u.empty()) {
            int u = stk_u.back();
            uint32_t e = stk_e.back();
            if (!e) {
                stk_u.pop_back();
                stk_e.pop_back();
                if (!stk_u.empty()) {
                    int p = stk_u.back();
                    if (low[u] >= disc[p]) {
                        int size = 1, w;
                        do {
                            w = vstk.back();
                            vstk.pop_back();
                            size++;
                        } while (w != u);
                        best = std::max(best, size);
                    }
                    low[p] = std::min(low[p], low[u]);
                }
                continue;
            }
            int v = __builtin_ffs((int)e) - 1;
            stk_e.back() = e & ~(1u << v);
            if (disc[v] < 0) {
                parent[v] = u;
                disc[v] = low[v] = t++;
                vstk.push_back(v);
                stk_u.push_back(v);
                stk_e.push_back(adj[v]);
            } else if (v != parent[u]) {
                low[u] = std::min(low[u], disc[v]);
            }
        }
        vstk.clear();
    }
    return best;
}

std::vector<uint32_t> build_blob(const HostInfo &info) {
    const int n_ec = (int)info.ec_relids.size();
    const int n_sels = (int)info.ec_sels.size();
    const int n_fks = (int)info.ec_fks.size();
    const int n = info.n;
    // tree-shaped query graph: n - 1 edges, connected
    int n_edges = 0;
    for (int i = 0; i < n; i++) n_edges += popc64(info.edge[i]);
    n_edges /= 2;
    bool tree = (n_edges == n - 1);
    if (tree) {
        mask64 seen = 1, frontier = 1;
        while (frontier) {
            mask64 next = 0;
            for (int i = 0; i < n; i++)
                if (frontier & bit64(i)) next |= info.edge[i] >> 1;
            frontier = next & ~seen;
            seen |= next;
        }
        tree = (seen == (n == 64 ? ~0ull : (bit64(n) - 1)));
    }
    const uint32_t base_words = blob_words_for(n, n_ec, n_sels, n_fks);
    std::vector<uint32_t> blob(base_words + (tree ? tree_tab_words(n) : 0u), 0u);
    DevHeader *h = reinterpret_cast<DevHeader *>(blob.data());
    h->n = n;
    h->n_ec = n_ec;
    h->n_sels = n_sels;
    h->n_fks = n_fks;
    h->cpu_operator_cost = info.p.cpu_operator_cost;
    h->cpu_tuple_cost = info.p.cpu_tuple_cost;
    h->seq_page_cost = info.p.seq_page_cost;
    h->disable_cost = info.p.disable_cost;
    h->work_mem = info.p.work_mem;
    h->enable_nestloop = info.p.enable_nestloop ? 1 : 0;
    h->enable_hashjoin = info.p.enable_hashjoin ? 1 : 0;
    h->composite_mask = 0;
    h->blob_words = (uint32_t)blob.size();
    // every biconnected block of a tree is one edge
    h->max_block = tree ? (uint32_t)std::min(n, 2) : (uint32_t)max_block_size(info);
    long long width_sum = 0;
    bool width_ok = true;
    for (int i = 0; i < n; i++) {
        width_sum += info.base[i].width;
        width_ok = width_ok && info.base[i].width >= 0;
    }
    h->hz_packed = (width_ok && width_sum < (1ll << 21)) ? 1u : 0u;   // kWidthBits
    for (int i = 0; i < n; i++) {
        h->adj[i] = (uint32_t)(info.edge[i] >> 1);
        h->rows[i] = info.base[i].rows;
        h->tuples[i] = info.base[i].tuples;
        h->startup[i] = info.base[i].cost.startup;
        h->total[i] = info.base[i].cost.total;
        h->width[i] = info.base[i].width;
        h->fksel[i] = (float)(1.0 / (double)std::fmax(1.0f, info.base[i].tuples));
        if (info.base[i].composite) h->composite_mask |= 1u << i;
    }
    h->tree_mode = tree ? 1u : 0u;
    h->ec_masked = 0u;
    h->tree_tab = 0u;
    if (tree) {
        h->tree_tab = base_words;
        uint32_t *tab = blob.data() + base_words;
        const int nn = n * n;
        uint32_t adj[32];
        for (int v = 0; v < n; v++) adj[v] = h->adj[v];
        for (int r = 0; r < n; r++) {
            // The kernels read the rows of root r only for sets whose lowest
            // relation is r (and row 0 for the classes on edges): a relation
            // without a higher-numbered neighbour is never the lowest of a
            // connected set of two or more, and its rows stay zero.
            if (r > 0 && (adj[r] >> r) <= 1u) continue;
            // preorder from r, children in increasing index order (pushed from
            // the highest index, so the lowest is visited first); n <= 32, so
            // fixed arrays
            uint32_t par_bit[32], anc[32], sub[32], before_of[32];
            int order[32], stack[32];
            int sp = 0, no = 0;
            anc[r] = 0u;
            par_bit[r] = 0u;
            stack[sp++] = r;
            uint32_t before = 0u;
            while (sp > 0) {
                const int u = stack[--sp];
                before_of[u] = before;
                before |= 1u << u;
                order[no++] = u;
                uint32_t kids = adj[u] & ~par_bit[u];
                const uint32_t anc_kid = anc[u] | (1u << u);
                while (kids) {
                    const int c = 31 - __builtin_clz(kids);
                    kids &= ~(1u << c);
                    par_bit[c] = 1u << u;
                    anc[c] = anc_kid;
                    stack[sp++] = c;
                }
            }
            for (int v = 0; v < n; v++) sub[v] = 1u << v;
            for (int i = no - 1; i > 0; i--) sub[__builtin_ctz(par_bit[order[i]])] |= sub[order[i]];
            std::memcpy(tab + r * n, sub, (size_t)n * 4u);
            std::memcpy(tab + nn + r * n, before_of, (size_t)n * 4u);
            std::memcpy(tab + 2 * nn + r * n, anc, (size_t)n * 4u);
        }
        // classes on edges: every 2-member class must sit on an edge
        bool masked = n_ec <= 32;
        for (int e = 0; masked && e < n_ec; e++) {
            uint32_t rr = (uint32_t)(info.ec_relids[e] >> 1);
            if (popc64(rr) != 2) {
                masked = false;
                break;
            }
            int a = __builtin_ctz(rr), b = 31 - __builtin_clz(rr);
            if (!((h->adj[a] >> b) & 1u)) {
                masked = false;   // a class between relations that are not adjacent
                break;
            }
            int child0 = ((tab[2 * nn + 0 * n + b] >> a) & 1u) ? b : a;
            h->edge_ec[child0] |= 1u << e;
        }
        if (masked) h->ec_masked = 1u;
        else
            for (int i = 0; i < n; i++) h->edge_ec[i] = 0u;
    }
    DevInfoView v = make_view(blob.data());
    uint32_t *relids = const_cast<uint32_t *>(v.ec_relids);
    uint32_t *offs = const_cast<uint32_t *>(v.ec_off);
    float *sels = const_cast<float *>(v.sels);
    uint32_t *fks = const_cast<uint32_t *>(v.fks);
    DevVar *vars = const_cast<DevVar *>(v.vars);
    int off_sels = 0, off_fks = 0;
    for (int i = 0; i < n_ec; i++) {
        relids[i] = (uint32_t)(info.ec_relids[i] >> 1);
        offs[i] = ((uint32_t)off_sels << 16) | (uint32_t)off_fks;
        // member j of the class (in relation order) owns fks/vars[off_fks + j]
        mask64 m = info.ec_relids[i] >> 1;
        for (int j = 0; m; j++, m &= m - 1) {
            const int rel = __builtin_ctzll(m);
            const int f = off_fks + j;
            fks[f] = (uint32_t)(info.ec_fks[f] >> 1);
            const VarInfo &vi = info.ec_vars[f];
            vars[f].idx_rows = vi.index.rows;
            vars[f].idx_startup = vi.index.cost.startup;
            vars[f].idx_total = vi.index.cost.total;
            vars[f].flags = (vi.index.available ? 1u : 0u) | (vi.index.unique ? 2u : 0u);
            devvar_bucket_terms(vars[f], vi.stats.stadistinct, vi.stats.stanullfrac, vi.stats.mcvfreq, h->rows[rel],
                                h->tuples[rel]);
        }
        int s = popc64(info.ec_relids[i]);
        off_sels += ec_nsels(s);
        off_fks += s;
    }
    for (int i = 0; i < n_sels; i++) sels[i] = info.ec_sels[i];
    fill_rel_ecs(v, n);
    fill_pair_sel(v);
    if (h->ec_masked) {
        // ec_selectivity (gpuqo_row_estimation.cuh:49-88) of each two-member
        // class in both orientations: the FK selectivity of the outer member's
        // key into the inner member, else the reverse key, else sels[0]
        for (int i = 0; i < n_ec; i++) {
            const uint32_t rr = relids[i];
            const int x = __builtin_ctz(rr), y = 31 - __builtin_clz(rr);
            const int off_f = (int)(offs[i] & 0xFFFFu), off_s = (int)(offs[i] >> 16);
            const bool fk_xy = (fks[off_f + 0] >> y) & 1u;   // member x's key matches y
            const bool fk_yx = (fks[off_f + 1] >> x) & 1u;   // member y's key matches x
            const float s = sels[off_s];
            h->edge_sel[0][i] = fk_xy ? h->fksel[y] : (fk_yx ? h->fksel[x] : s);
            h->edge_sel[1][i] = fk_yx ? h->fksel[x] : (fk_xy ? h->fksel[y] : s);
        }
    }
    return blob;
}

bool use_sparse_memo(int n, DpMode mode) {
    if (n > 31) return true;
    const int from = gpuqo_b200_sparse_from_rels;
    return from > 0 && from < 32 && n >= from && mode != kModeDpsize;
}

// Exact DP of a relabelled info on the GPU: up to 31 relations with the dense
// memo, 32 to 63 with the sparse memo of the connected sets (dp_wide.cu).
int exact_dp(const HostInfo &info, DpMode mode, std::vector<TreeNode> &nodes, std::string &err) {
    if (info.n > 63) {
        err = "exact DP over " + std::to_string(info.n) + " relations exceeds the 64-bit relation sets";
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    if (use_sparse_memo(info.n, mode)) {
        EngineStats st;
        const int rc = engine_run_wide(info, mode, nodes, st, err);
        if (rc == 0) stats_add(st);
        return rc;
    }
    if (info.ec_sels.size() >= 65536 || info.ec_fks.size() >= 65536) {
        err = "too many equivalence-class entries";
        return GPUQO_B200_ERR_ARGS;
    }
    std::vector<uint32_t> blob = build_blob(info);
    apply_dpsub_csg(blob, mode);
    EngineStats st;
    int rc = engine_run(blob, info.n, mode, gpuqo_dpsub_ccc_enable, gpuqo_b200_profile_kernels != 0, nodes, st, err);
    if (rc == 0) stats_add(st);
    return rc;
}

void apply_dpsub_csg(std::vector<uint32_t> &blob, DpMode &mode) {
    if (mode != kModeDpsub || !gpuqo_dpsub_csg_enable) return;
    DevHeader *h = reinterpret_cast<DevHeader *>(blob.data());
    // On a dense graph nearly every subset is a valid split, so the block
    // enumeration saves nothing and only adds the index computation: keep
    // the all-subsets enumeration at or above half of all possible edges.
    // Either enumeration returns the same plan.
    uint64_t degree_sum = 0;
    for (int i = 0; i < h->n; i++) degree_sum += (uint64_t)__builtin_popcount(h->adj[i]);
    if (2 * degree_sum >= (uint64_t)h->n * (uint64_t)(h->n - 1)) return;
    h->index_order = 1u;
    mode = kModeMpdp;
}

DpMode mode_for(int algorithm) {
    switch (algorithm) {
    case GPUQO_DPSIZE:
    case GPUQO_CPU_DPSIZE:
    case GPUQO_DPE_DPSIZE:
        return kModeDpsize;
    case GPUQO_CPU_DPSUB_BICC:
    case GPUQO_CPU_DPSUB_BICC_PARALLEL:
        return kModeMpdp;
    case GPUQO_CPU_DPSUB:
    case GPUQO_CPU_DPSUB_PARALLEL:
    case GPUQO_DPE_DPSUB:
        return kModeDpsub;
    default:
        return gpuqo_dpsub_bicc_enable ? kModeMpdp : kModeDpsub;
    }
}

bool algorithm_supported(int algorithm) {
    switch (algorithm) {
    case GPUQO_DPSIZE:
    case GPUQO_CPU_DPSIZE:
    case GPUQO_DPE_DPSIZE:
    case GPUQO_DPSUB:
    case GPUQO_CPU_DPSUB:
    case GPUQO_CPU_DPSUB_PARALLEL:
    case GPUQO_CPU_DPSUB_BICC:
    case GPUQO_CPU_DPSUB_BICC_PARALLEL:
    case GPUQO_DPE_DPSUB:
        return true;
    default:
        return false;
    }
}

static Bitmapset *make_bms(mask64 m) {
    Bitmapset *b = (Bitmapset *)palloc0(offsetof(Bitmapset, words) + sizeof(bitmapword));
    b->nwords = 1;
    b->words[0] = m;
    return b;
}

// node array (compact masks over relabelled relations) -> QueryTreeC with the
// caller's relids (remapQueryTree gpuqo_remapper.cu:279-300, convertQueryTree
// gpuqo_planner_info.cu:256-270)
static QueryTreeC *nodes_to_c(const std::vector<TreeNode> &nodes, int idx, const std::vector<int> &from_of_to) {
    if (idx < 0) return NULL;
    const TreeNode &t = nodes[idx];
    QueryTreeC *q = (QueryTreeC *)palloc(sizeof(QueryTreeC));
    mask64 orig = 0;
    for (uint64_t x = t.set; x; x &= x - 1ull) orig |= bit64(from_of_to[__builtin_ctzll(x)] + 1);
    q->id = make_bms(orig);
    q->left = nodes_to_c(nodes, t.left, from_of_to);
    q->right = nodes_to_c(nodes, t.right, from_of_to);
    q->width = t.width;
    q->cost.startup = t.startup;
    q->cost.total = t.total;
    q->rows = t.rows;
    return q;
}

static double g_tune_ms = 0.0;

QueryTreeC *run_one(int algorithm, GpuqoPlannerInfoC *info_c) {
    t_last_error = GPUQO_B200_OK;
    std::string err;
    if (!algorithm_supported(algorithm)) {
        set_error(GPUQO_B200_ERR_UNSUPPORTED,
                  "algorithm " + std::to_string(algorithm) + " is outside this library (DPsub/MPDP only)");
        return NULL;
    }
    if (!info_c || info_c->n_rels < 1) {
        set_error(GPUQO_B200_ERR_ARGS, "empty planner info");
        return NULL;
    }
    if (InterruptPending) {
        ProcessInterrupts();
        set_error(GPUQO_B200_ERR_CANCELLED, "cancelled");
        return NULL;
    }
    const int n = info_c->n_rels;
    const bool idp = gpuqo_idp_n_iters > 1 && gpuqo_idp_n_iters < n;
    if (idp || n >= 64 || gpuqo_spanning_tree_enable) return run_planned(algorithm, info_c);

    HostInfo info;
    if (!convert_info(info_c, info, err)) {
        set_error(GPUQO_B200_ERR_ARGS, err);
        return NULL;
    }
    std::vector<int> order = bfs_order(info);
    if ((int)order.size() != info.n) {
        // the reference plans connected query graphs only (a join tree of a
        // BFS order that misses relations would lose them)
        set_error(GPUQO_B200_ERR_ARGS, "query graph is not connected");
        return NULL;
    }
    HostInfo remapped = relabel(info, order);
    std::vector<TreeNode> nodes;
    int rc = exact_dp(remapped, mode_for(algorithm), nodes, err);
    if (rc) {
        set_error(rc, err);
        return NULL;
    }
    return nodes_to_c(nodes, 0, order);
}

}  // namespace gqb

using namespace gqb;

extern "C" QueryTreeC *gpuqo_run(int gpuqo_algorithm_arg, GpuqoPlannerInfoC *info) {
    stats_reset();
    return run_one(gpuqo_algorithm_arg, info);
}

extern "C" int gpuqo_b200_last_error(void) { return t_last_error; }

extern "C" void gpuqo_b200_free_query_tree(QueryTreeC *qt) {
    if (!qt) return;
    gpuqo_b200_free_query_tree(qt->left);
    gpuqo_b200_free_query_tree(qt->right);
    if (qt->id) pfree(qt->id);
    pfree(qt);
}

extern "C" void gpuqo_b200_get_stats(GpuqoB200Stats *out) {
    if (out) *out = t_stats;
}

extern "C" int gpuqo_b200_time_resident(int gpuqo_algorithm_arg, GpuqoPlannerInfoC *info_c, int warmup, int iters,
                                        int flush_l2, double *ms_per_iter, QueryTreeC **tree) {
    stats_reset();
    t_last_error = GPUQO_B200_OK;
    std::string err;
    if (!algorithm_supported(gpuqo_algorithm_arg) || !info_c || info_c->n_rels < 1 || info_c->n_rels > 31 ||
        warmup < 0 || iters < 1 || !ms_per_iter) {
        set_error(GPUQO_B200_ERR_ARGS, "gpuqo_b200_time_resident: bad arguments");
        return t_last_error;
    }
    if (gpuqo_spanning_tree_enable) {
        set_error(GPUQO_B200_ERR_UNSUPPORTED, "gpuqo_b200_time_resident times the query graph as given "
                                              "(gpuqo_spanning_tree_enable is set)");
        return t_last_error;
    }
    HostInfo info;
    if (!convert_info(info_c, info, err)) {
        set_error(GPUQO_B200_ERR_ARGS, err);
        return t_last_error;
    }
    std::vector<int> order = bfs_order(info);
    if ((int)order.size() != info.n) {
        set_error(GPUQO_B200_ERR_ARGS, "query graph is not connected");
        return t_last_error;
    }
    HostInfo remapped = relabel(info, order);
    std::vector<uint32_t> blob = build_blob(remapped);
    DpMode mode = mode_for(gpuqo_algorithm_arg);
    apply_dpsub_csg(blob, mode);
    std::vector<TreeNode> nodes;
    EngineStats st;
    int rc = engine_time_resident(blob, remapped.n, mode, gpuqo_dpsub_ccc_enable, warmup, iters, flush_l2 != 0,
                                  *ms_per_iter, nodes, st, err);
    if (rc) {
        set_error(rc, err);
        return rc;
    }
    stats_add(st);
    if (tree) *tree = nodes_to_c(nodes, 0, order);
    return GPUQO_B200_OK;
}

// A seeded star of n relations in the shape of the synthetic workloads: fact
// table 1e7 rows, dimensions log-uniform in [1e2, 1e5], FK-PK classes.
static HostInfo synthetic_star(int n, uint32_t seed) {
    HostInfo h;
    h.n = n;
    h.p = read_params();
    uint32_t x = seed * 2654435761u + 12345u;
    auto uniform = [&]() {
        x ^= x << 13;
        x ^= x >> 17;
        x ^= x << 5;
        return (float)(x & 0xFFFFFFu) / 16777216.0f;
    };
    for (int i = 0; i < n; i++) {
        HostBaseRel b{};
        b.id = bit64(i + 1);
        b.rows = i == 0 ? 1e7f : std::floor(100.0f * std::pow(1000.0f, uniform()));
        b.tuples = b.rows;
        b.width = 8;
        b.cost.startup = 0.0f;
        b.cost.total = b.rows * 0.01f;
        b.composite = false;
        h.base.push_back(b);
    }
    h.edge.assign(n, 0);
    for (int i = 1; i < n; i++) {
        h.edge[0] |= bit64(i + 1);
        h.edge[i] |= bit64(1);
        h.ec_relids.push_back(bit64(1) | bit64(i + 1));
        h.ec_sels.push_back(1.0f / h.base[i].rows);
        h.ec_fks.push_back(bit64(i + 1));   // the fact's key references dimension i
        h.ec_fks.push_back(0);
        h.ec_vars.push_back(VarInfo{});
        h.ec_vars.push_back(VarInfo{});
    }
    return h;
}

extern "C" int gpuqo_b200_autotune(GpuqoB200Tuning *out) {
    t_last_error = GPUQO_B200_OK;
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::vector<uint32_t>> blobs;
    for (int n : {14, 16, 18, 19, 20, 21, 22, 23, 24}) blobs.push_back(build_blob(synthetic_star(n, 7u + n)));
    double narrow = 0.0, wide = 0.0, single = 0.0;
    std::string err;
    if (int rc = engine_autotune(blobs, narrow, wide, single, err)) {
        set_error(rc, err);
        return rc;
    }
    g_tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return gpuqo_b200_get_tuning(out);
}

extern "C" int gpuqo_b200_reset_persistent(void) { return engine_reset_persistent(); }

extern "C" int gpuqo_b200_set_tuning(const GpuqoB200Tuning *in) {
    if (!in) return GPUQO_B200_ERR_ARGS;
    for (double v : {in->single_narrow_level_sets, in->single_wide_level_sets, in->batch_single_sets})
        if (!(v >= 0.0)) return GPUQO_B200_ERR_ARGS;   // negative or NaN
    engine_set_tuning(in->single_narrow_level_sets, in->single_wide_level_sets, in->batch_single_sets,
                      in->tuned != 0);
    return GPUQO_B200_OK;
}

extern "C" int gpuqo_b200_get_tuning(GpuqoB200Tuning *out) {
    if (!out) return GPUQO_B200_ERR_ARGS;
    bool tuned = false;
    engine_get_tuning(out->single_narrow_level_sets, out->single_wide_level_sets, out->batch_single_sets, tuned);
    out->tuned = tuned ? 1 : 0;
    out->tune_ms = tuned ? g_tune_ms : 0.0;
    return GPUQO_B200_OK;
}

namespace gqb {

// Longest-processing-time assignment of weighted work items to n_dev devices:
// items in decreasing weight (lower index first on ties), each to the device
// with the least weight so far (lower index first on ties).  Deterministic;
// every device gets items before any gets a second when there are enough.
void plan_shards(const double *work, int n, int n_dev, int *dev_of) {
    if (n_dev < 1) n_dev = 1;
    std::vector<int> order((size_t)n);
    for (int i = 0; i < n; i++) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::vector<double> load((size_t)n_dev, 0.0);
    for (int i : order) {
        int best = 0;
        for (int d = 1; d < n_dev; d++)
            if (load[(size_t)d] < load[(size_t)best]) best = d;
        dev_of[i] = best;
        load[(size_t)best] += work[i];
    }
}

// gpuqo_b200_devices: 1 (default) the calling thread's current device; N > 1
// the N devices from the current one on (wrapping around the visible ones);
// 0 every visible device, the current one first
int batch_devices(std::vector<int> &devs, std::string &err) {
    int cur = 0, count = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (e == cudaSuccess) e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        err = std::string("device query: ") + cudaGetErrorString(e);
        return GPUQO_B200_ERR_CUDA;
    }
    const int want = gpuqo_b200_devices <= 0 ? count : gpuqo_b200_devices;
    devs.clear();
    for (int j = 0; j < std::max(want, 1); j++) devs.push_back((cur + j) % std::max(count, 1));
    return 0;
}

}  // namespace gqb

extern "C" int gpuqo_b200_plan_shards(const double *work, int n_items, int n_devices, int *device_of_item) {
    if (!work || !device_of_item || n_items < 0 || n_devices < 1) return GPUQO_B200_ERR_ARGS;
    plan_shards(work, n_items, n_devices, device_of_item);
    return GPUQO_B200_OK;
}

extern "C" int gpuqo_b200_run_batch(int gpuqo_algorithm_arg, GpuqoPlannerInfoC **infos, int n_queries,
                                    QueryTreeC **out) {
    stats_reset();
    t_last_error = GPUQO_B200_OK;
    if (!infos || !out || n_queries < 0) return GPUQO_B200_ERR_ARGS;
    for (int i = 0; i < n_queries; i++) out[i] = NULL;
    if (!algorithm_supported(gpuqo_algorithm_arg)) {
        set_error(GPUQO_B200_ERR_UNSUPPORTED, "algorithm outside this library");
        return GPUQO_B200_ERR_UNSUPPORTED;
    }
    const DpMode mode = mode_for(gpuqo_algorithm_arg);
    // Prepare every query as gpuqo_run does (convert, BFS relabel); MPDP
    // queries without IDP whose candidate count fits the batched kernel go to
    // the level-synchronous batch, the rest run one by one.
    struct Prep {
        std::vector<int> order;
        std::vector<uint32_t> blob;
    };
    std::vector<Prep> prep(n_queries);
    std::vector<char> to_batch(n_queries, 0);
    // reads the caller's structures and allocates with malloc only (no
    // palloc), so the queries are prepared on several host threads
    auto prepare = [&](int i) {
        GpuqoPlannerInfoC *c = infos[i];
        const bool idp = c && gpuqo_idp_n_iters > 1 && gpuqo_idp_n_iters < c->n_rels;
        // the planner path (run_one) applies gpuqo_spanning_tree_enable
        if (!c || c->n_rels < 1 || c->n_rels > 30 || idp || gpuqo_spanning_tree_enable) return;
        DpMode m = mode;
        HostInfo info;
        std::string err;
        if (!convert_info(c, info, err)) return;
        prep[i].order = bfs_order(info);
        if ((int)prep[i].order.size() != info.n) return;
        HostInfo remapped = relabel(info, prep[i].order);
        prep[i].blob = build_blob(remapped);
        apply_dpsub_csg(prep[i].blob, m);
        to_batch[i] = (m == kModeMpdp && batch_eligible(prep[i].blob)) ? 1 : 0;
    };
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int n_threads = n_queries >= 64 ? std::min({hw, 16, n_queries / 32}) : 1;
    if (n_threads > 1) {
        std::vector<std::thread> pool;
        for (int t = 0; t < n_threads; t++)
            pool.emplace_back([&, t] {
                for (int i = t; i < n_queries; i += n_threads) prepare(i);
            });
        for (auto &th : pool) th.join();
    } else {
        for (int i = 0; i < n_queries; i++) prepare(i);
    }
    std::vector<int> batched, single;
    for (int i = 0; i < n_queries; i++) (to_batch[i] ? batched : single).push_back(i);
    int status = GPUQO_B200_OK;
    if (!batched.empty()) {
        // larger queries first: a wave then runs only the levels it needs
        std::stable_sort(batched.begin(), batched.end(), [&](int a, int b) {
            return infos[a]->n_rels > infos[b]->n_rels;
        });
        const uint64_t budget = (uint64_t)std::max(gpuqo_b200_batch_memory_mb, 64) << 20;
        // the devices the batch is spread over (gpuqo_b200_devices), and each
        // query's device by estimated work (longest first, least loaded)
        std::vector<int> devs;
        std::string err;
        if (int rc = batch_devices(devs, err)) {
            set_error(rc, err);
            return rc;
        }
        std::vector<double> work(batched.size());
        for (size_t j = 0; j < batched.size(); j++) work[j] = engine_work_estimate(prep[batched[j]].blob);
        std::vector<int> shard(batched.size(), 0);
        plan_shards(work.data(), (int)work.size(), (int)devs.size(), shard.data());
        std::vector<std::vector<TreeNode>> nodes(batched.size());
        std::vector<EngineStats> dst(devs.size());
        std::vector<int> drc(devs.size(), 0);
        std::vector<std::string> derr(devs.size());
        // one host thread per device with queries; each runs its own waves
        // on its own engines (queries keep their largest-first order)
        auto run_shard = [&](size_t d) {
            std::vector<const std::vector<uint32_t> *> blobs;
            std::vector<size_t> idx;
            for (size_t j = 0; j < batched.size(); j++)
                if (shard[j] == (int)d) {
                    blobs.push_back(&prep[batched[j]].blob);
                    idx.push_back(j);
                }
            if (blobs.empty()) return;
            if (devs.size() > 1) {
                const cudaError_t e = cudaSetDevice(devs[d]);
                if (e != cudaSuccess) {
                    cudaGetLastError();
                    drc[d] = GPUQO_B200_ERR_CUDA;
                    derr[d] = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
                    return;
                }
            }
            std::vector<std::vector<TreeNode>> dn;
            std::vector<double> wave_ms;
            drc[d] = engine_run_batch(blobs, budget, dn, dst[d], wave_ms, derr[d]);
            if (!drc[d])
                for (size_t q = 0; q < idx.size(); q++) nodes[idx[q]] = std::move(dn[q]);
        };
        if (devs.size() == 1) {
            run_shard(0);
        } else {
            std::vector<std::thread> th;
            for (size_t d = 0; d < devs.size(); d++) th.emplace_back(run_shard, d);
            for (auto &t : th) t.join();
        }
        EngineStats st;
        for (size_t d = 0; d < devs.size(); d++) {
            if (drc[d]) {
                set_error(drc[d], derr[d]);
                return drc[d];
            }
            st.connected_sets += dst[d].connected_sets;
            st.evaluated_pairs += dst[d].evaluated_pairs;
            st.memo_bytes = std::max(st.memo_bytes, dst[d].memo_bytes);
            st.device_ms = std::max(st.device_ms, dst[d].device_ms);   // devices run side by side
            st.kernel_launches += dst[d].kernel_launches;
            st.barrier_timeouts += dst[d].barrier_timeouts;
            st.handoff_ms += dst[d].handoff_ms;
        }
        stats_add(st);
        t_stats.n_subproblems = (uint32_t)batched.size();
        for (size_t j = 0; j < batched.size(); j++)
            out[batched[j]] = nodes_to_c(nodes[j], 0, prep[batched[j]].order);
    }
    for (int i : single) {
        out[i] = run_one(gpuqo_algorithm_arg, infos[i]);
        if (!out[i]) status = t_last_error;
    }
    return status;
}
