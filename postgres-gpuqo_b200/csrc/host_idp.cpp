// host_idp.cpp - IDP2 and UnionDP drivers over the GPU exact DP.
//
// Restates, on the host, the reference's iterative drivers and the machinery
// they use, for queries of any size (relations up to kBigBits - 1):
//   gpuqo_run_idp2 / _rec / find_most_expensive_subtree  gpuqo_idp.cu:96-297
//   gpuqo_run_dpdp_union / _rec, DisjointSet, edge queues gpuqo_dpdp_union.cu:29-472
//   gpuqo_cpu_goo (IDP2's seed plan)                      gpuqo_cpu_goo.cu:27-150
//   Remapper (composite relations, re-estimated classes)  gpuqo_remapper.cu:34-300
//   makeBFSIndexRemapper                                   gpuqo_bfs_indexing.cu:14-55
//   estimate_join_rows/selectivity on plan nodes           gpuqo_row_estimation.cuh:26-148
// Every sub-problem (at most 63 relations after remapping; above 31 on the
// sparse memo) is solved by the GPU engine through exact_dp(), without a BFS
// relabelling, as the reference calls gpuqo_run_switch on the remapped info.
//
// The remapper's lookups, which the reference performs by scanning its list
// of entries, use an owner table instead (entries partition the relations,
// so "entry e intersects id" is "some relation of id is owned by e"); results
// are identical.  The heaps and priority queues are the same libstdc++
// algorithms fed in the same order, so their tie behaviour is the reference's.
#include <algorithm>
#include <limits>
#include <atomic>
#include <csignal>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <queue>
#include <string>
#include <vector>

#include "dp_engine.h"
#include "gpuqo_b200.h"
#include "host_idp.h"
#include "host_info.h"

extern "C" int gpuqo_idp_n_iters;
extern "C" int gpuqo_idp_type;
extern "C" bool gpuqo_spanning_tree_enable;
extern "C" volatile sig_atomic_t InterruptPending;
extern "C" void *palloc(size_t size);
extern "C" void *palloc0(size_t size);

namespace gqb {

int exact_dp(const HostInfo &info, DpMode mode, std::vector<TreeNode> &nodes, std::string &err);
DpMode mode_for(int algorithm);

// ---------------------------------------------------------------------------
// fixed-capacity bitset with the reference's numbering (relation i = bit i+1)
// ---------------------------------------------------------------------------
constexpr int kBigWords = 16;
constexpr int kBigBits = kBigWords * 64;

struct BB {
    std::array<uint64_t, kBigWords> w{};
    static BB bit(int i) {
        BB b;
        b.w[i >> 6] = 1ull << (i & 63);
        return b;
    }
    bool test(int i) const { return (w[i >> 6] >> (i & 63)) & 1ull; }
    void set(int i) { w[i >> 6] |= 1ull << (i & 63); }
    void unset(int i) { w[i >> 6] &= ~(1ull << (i & 63)); }
    bool empty() const {
        for (auto x : w)
            if (x) return false;
        return true;
    }
    int size() const {
        int c = 0;
        for (auto x : w) c += __builtin_popcountll(x);
        return c;
    }
    int lowest_pos() const {
        for (int i = 0; i < kBigWords; i++)
            if (w[i]) return i * 64 + __builtin_ctzll(w[i]);
        return -1;
    }
    BB lowest() const {
        BB b;
        int p = lowest_pos();
        if (p >= 0) b.set(p);
        return b;
    }
    // all bits below the lowest set bit (GpuqoBitmapset::allLower)
    BB all_lower() const {
        BB b;
        int p = lowest_pos();
        if (p < 0) return b;
        for (int i = 0; i < (p >> 6); i++) b.w[i] = ~0ull;
        if (p & 63) b.w[p >> 6] = (1ull << (p & 63)) - 1ull;
        return b;
    }
    BB operator|(const BB &o) const {
        BB r;
        for (int i = 0; i < kBigWords; i++) r.w[i] = w[i] | o.w[i];
        return r;
    }
    BB operator&(const BB &o) const {
        BB r;
        for (int i = 0; i < kBigWords; i++) r.w[i] = w[i] & o.w[i];
        return r;
    }
    BB operator-(const BB &o) const {
        BB r;
        for (int i = 0; i < kBigWords; i++) r.w[i] = w[i] & ~o.w[i];
        return r;
    }
    BB &operator|=(const BB &o) {
        for (int i = 0; i < kBigWords; i++) w[i] |= o.w[i];
        return *this;
    }
    BB &operator-=(const BB &o) {
        for (int i = 0; i < kBigWords; i++) w[i] &= ~o.w[i];
        return *this;
    }
    bool intersects(const BB &o) const {
        for (int i = 0; i < kBigWords; i++)
            if (w[i] & o.w[i]) return true;
        return false;
    }
    bool is_subset_of(const BB &o) const {
        for (int i = 0; i < kBigWords; i++)
            if (w[i] & ~o.w[i]) return false;
        return true;
    }
    bool operator==(const BB &o) const { return w == o.w; }
    bool operator!=(const BB &o) const { return w != o.w; }
    // integer order (Bitmapset32/64 compare bits; bms_compare compares from
    // the highest word down)
    bool operator<(const BB &o) const {
        for (int i = kBigWords - 1; i >= 0; i--)
            if (w[i] != o.w[i]) return w[i] < o.w[i];
        return false;
    }
    template <class F> void for_each(F f) const {
        for (int i = 0; i < kBigWords; i++) {
            uint64_t x = w[i];
            while (x) {
                f(i * 64 + __builtin_ctzll(x));
                x &= x - 1;
            }
        }
    }
};

struct GBase {
    BB id;
    float rows, tuples;
    int width;
    PathCost cost;
    bool composite;
};

// Lists of ints stored back to back (offsets + one array): list i is
// [data + off[i], data + off[i + 1]).  Indexing gives a view with begin/end/
// size, so callers read it like a vector of vectors without one allocation
// per list.
struct IntLists {
    std::vector<int> off{0}, data;
    struct View {
        const int *b, *e;
        const int *begin() const { return b; }
        const int *end() const { return e; }
        size_t size() const { return (size_t)(e - b); }
    };
    View operator[](size_t i) const { return View{data.data() + off[i], data.data() + off[i + 1]}; }
    size_t size() const { return off.size() - 1; }
};

struct GInfo {
    int n = 0;
    HostParams p;
    std::vector<GBase> base;
    std::vector<BB> edge;
    std::vector<BB> ec;                // relids
    IntLists ec_members;               // relation indices (bit - 1), increasing
    std::vector<float> sels;
    std::vector<BB> fks;
    std::vector<VarInfo> vars;
    std::vector<int> ec_off_sels, ec_off_fks;
    IntLists rel_ecs;                  // per relation: classes containing it, increasing
    void index() {
        const size_t n_ec = ec.size();
        ec_off_sels.assign(n_ec, 0);
        ec_off_fks.assign(n_ec, 0);
        ec_members.off.assign(n_ec + 1, 0);
        rel_ecs.off.assign((size_t)n + 1, 0);
        // counts, then offsets, then the members in class order
        int os = 0, of = 0;
        for (size_t i = 0; i < n_ec; i++) {
            int s = 0;
            ec[i].for_each([&](int b) {
                s++;
                if (b >= 1 && b - 1 < n) rel_ecs.off[b]++;
            });
            ec_members.off[i + 1] = ec_members.off[i] + s;
            ec_off_sels[i] = os;
            ec_off_fks[i] = of;
            os += s * (s - 1) / 2;
            of += s;
        }
        for (int r = 0; r < n; r++) rel_ecs.off[r + 1] += rel_ecs.off[r];
        ec_members.data.resize((size_t)ec_members.off[n_ec]);
        rel_ecs.data.resize((size_t)rel_ecs.off[n]);
        std::vector<int> fill(rel_ecs.off.begin(), rel_ecs.off.end() - 1);
        for (size_t i = 0; i < n_ec; i++) {
            int k = ec_members.off[i];
            ec[i].for_each([&](int b) {
                ec_members.data[k++] = b - 1;
                if (b >= 1 && b - 1 < n) rel_ecs.data[fill[b - 1]++] = (int)i;
            });
        }
    }
};

struct QT {
    BB id;
    float rows;
    PathCost cost;
    int width;
    QT *left = nullptr, *right = nullptr;
};

// node arena of one gpuqo_run call (the reference's trees are freed piecemeal;
// here they live until the call returns)
struct Arena {
    std::vector<std::unique_ptr<QT>> nodes;
    QT *make() {
        nodes.emplace_back(new QT());
        return nodes.back().get();
    }
};

static inline int ec_index(int l, int r, int size) {
    if (l > r) std::swap(l, r);
    return l * size - l * (l + 1) / 2 + (r - l - 1);
}

// ---------------------------------------------------------------------------
// row estimation on arbitrary relation sets (gpuqo_row_estimation.cuh)
// ---------------------------------------------------------------------------
static bool ec_hits(const GInfo &g, int e, const BB &s) {
    for (int m : g.ec_members[e])
        if (s.test(m + 1)) return true;
    return false;
}

// :26-45
static float fkselc_of_ec(const GInfo &g, int e, const BB &outer, const BB &inner) {
    BB tmp = outer;
    const BB &ecr = g.ec[e];
    while (!tmp.empty()) {
        BB out_id = tmp.lowest();
        int out_idx = (out_id.all_lower() & ecr).size();
        BB match = inner & g.fks[g.ec_off_fks[e] + out_idx];
        if (!match.empty()) {
            int in_idx = match.lowest_pos() - 1;
            return (float)(1.0 / (double)std::fmax(1.0f, g.base[in_idx].tuples));
        }
        tmp -= out_id;
    }
    return NAN;
}

// :49-88
static float estimate_ec_selectivity(const GInfo &g, int e, const BB &l, const BB &r) {
    const BB &ecr = g.ec[e];
    int size = (int)g.ec_members[e].size();
    if (size == 2) {
        // Two members m0 < m1: with one on each side the steps below reduce
        // to bit tests (the member's position in the class is 0 or 1, the FK
        // match is the other member, ec_index(0, 1, 2) = 0).  A member on
        // both sides takes the general path.
        const int m[2] = {g.ec_members[e].begin()[0], g.ec_members[e].begin()[1]};
        const int ml = (l.test(m[0] + 1) ? 1 : 0) | (l.test(m[1] + 1) ? 2 : 0);
        const int mr = (r.test(m[0] + 1) ? 1 : 0) | (r.test(m[1] + 1) ? 2 : 0);
        if (!(ml & mr)) {
            if (!ml || !mr) return 1.0f;
            const int ia = ml == 1 ? 0 : 1, ib = 1 - ia;   // positions of the l-side and r-side members
            const int a = m[ia], b = m[ib];
            const int off = g.ec_off_fks[e];
            if (g.fks[off + ia].test(b + 1)) return (float)(1.0 / (double)std::fmax(1.0f, g.base[b].tuples));
            if (g.fks[off + ib].test(a + 1)) return (float)(1.0 / (double)std::fmax(1.0f, g.base[a].tuples));
            return g.sels[g.ec_off_sels[e]];
        }
    }
    BB ml = ecr & l, mr = ecr & r;
    if (ml.empty() || mr.empty()) return 1.0f;
    float fk = fkselc_of_ec(g, e, ml, mr);
    if (!std::isnan(fk)) return fk;
    fk = fkselc_of_ec(g, e, mr, ml);
    if (!std::isnan(fk)) return fk;
    int il = (ml.all_lower() & ecr).size();
    int ir = (mr.all_lower() & ecr).size();
    return g.sels[g.ec_off_sels[e] + ec_index(il, ir, size)];
}

// :93-118.  Only classes with a member on both sides contribute a factor
// other than 1.0f; they are found through the smaller side's relations and
// multiplied in increasing class order, as the reference's loop does.
static float estimate_join_selectivity(const GInfo &g, const BB &l, const BB &r) {
    const BB &small = (l.size() <= r.size()) ? l : r;
    const BB &other = (&small == &l) ? r : l;
    thread_local std::vector<int> hit;   // reused: planners run on several threads
    hit.clear();
    small.for_each([&](int b) {
        if (b - 1 >= g.n) return;
        for (int e : g.rel_ecs[b - 1])
            if (ec_hits(g, e, other)) hit.push_back(e);
    });
    std::sort(hit.begin(), hit.end());
    hit.erase(std::unique(hit.begin(), hit.end()), hit.end());
    float sel = 1.0f;
    for (int e : hit) sel *= estimate_ec_selectivity(g, e, l, r);
    return sel;
}

// :135-148 (QueryTree overload)
static float estimate_join_rows(const GInfo &g, const QT &l, const QT &r) {
    float sel = estimate_join_selectivity(g, l.id, r.id);
    float rows = sel * l.rows * r.rows;
    return rows > 1 ? std::round(rows) : 1;
}

// ---------------------------------------------------------------------------
// gpuqo_spanning_tree_enable (minimumSpanningTree, gpuqo_spanning_tree.cu:19-72,
// applied by __gpuqo_run before the BFS relabelling for every algorithm,
// gpuqo_main_internal.cu:94-100): the join graph is replaced by a spanning
// tree grown from relation 0, each step adding the edge from the tree to a
// new relation whose two base relations give the fewest estimated join rows
// (the first strict minimum, tree relations and their neighbours both in
// increasing order).  The equivalence classes stay as they are, so joins are
// still costed with every class; only the csg-cmp pairs follow the tree.
// A step that finds no edge with fewer rows than FLT_MAX (every estimate
// infinite or NaN; the reference leaves that case undefined) takes the first
// edge it visited.
// ---------------------------------------------------------------------------
static void spanning_tree(GInfo &g) {
    const int n = g.n;
    std::vector<BB> out(n);
    std::vector<char> in_tree(n, 0);
    BB S = BB::bit(1);
    in_tree[0] = 1;
    for (int added = 1; added < n; added++) {
        float best = std::numeric_limits<float>::max();
        int ai = -1, ao = -1, fi = -1, fo = -1;
        for (int i = 0; i < n; i++) {
            if (!in_tree[i]) continue;
            (g.edge[i] - S).for_each([&](int b) {
                const int j = b - 1;
                if (j < 0 || j >= n) return;
                if (fi < 0) {
                    fi = i;
                    fo = j;
                }
                const float sel = estimate_join_selectivity(g, BB::bit(i + 1), BB::bit(j + 1));
                const float r = sel * g.base[i].rows * g.base[j].rows;
                const float rows = r > 1 ? std::round(r) : 1;
                if (rows < best) {
                    best = rows;
                    ai = i;
                    ao = j;
                }
            });
        }
        if (ao < 0) {
            if (fo < 0) break;   // disconnected: refused by the caller's BFS check
            ai = fi;
            ao = fo;
        }
        S.set(ao + 1);
        in_tree[ao] = 1;
        out[ai].set(ao + 1);
        out[ao].set(ai + 1);
    }
    g.edge = std::move(out);
}

// ---------------------------------------------------------------------------
// conversion and relabelling
// ---------------------------------------------------------------------------
static BB bms_to_bb(const Bitmapset *b, bool &too_wide) {
    BB r;
    if (!b) return r;
    for (int i = 0; i < b->nwords; i++) {
        if (i >= kBigWords) {
            if (b->words[i]) too_wide = true;
            continue;
        }
        r.w[i] = b->words[i];
    }
    return r;
}

static bool convert_big(const GpuqoPlannerInfoC *c, GInfo &g, std::string &err) {
    if (c->n_rels >= kBigBits - 1) {
        err = "more than " + std::to_string(kBigBits - 2) + " relations";
        return false;
    }
    bool wide = false;
    g.n = c->n_rels;
    g.p = read_params();
    g.base.resize(g.n);
    g.edge.resize(g.n);
    for (int i = 0; i < g.n; i++) {
        g.edge[i] = bms_to_bb(c->edge_table[i], wide);
        GBase &b = g.base[i];
        b.id = bms_to_bb(c->base_rels[i].id, wide);
        b.rows = c->base_rels[i].rows;
        b.tuples = c->base_rels[i].tuples;
        b.width = c->base_rels[i].width;
        b.cost = c->base_rels[i].cost;
        b.composite = false;
        if (b.id != BB::bit(i + 1)) {
            err = "base relation " + std::to_string(i) + " does not carry relid bit " + std::to_string(i + 1);
            return false;
        }
    }
    for (const EqClassInfo *ec = c->eq_classes; ec; ec = ec->next) {
        BB r = bms_to_bb(ec->relids, wide);
        g.ec.push_back(r);
        int s = r.size();
        for (int j = 0; j < s * (s - 1) / 2; j++) g.sels.push_back(ec->sels[j]);
        for (int j = 0; j < s; j++) {
            g.fks.push_back(ec->fk ? bms_to_bb(ec->fk[j], wide) : BB());
            g.vars.push_back(ec->vars[j]);
        }
    }
    if (wide) {
        err = "relation ids beyond the supported range";
        return false;
    }
    g.index();
    return true;
}

struct Entry {
    BB from;
    int to;
    QT *qt;
};

// Remapper (gpuqo_remapper.cu) over a list of disjoint entries.
class Remap {
public:
    std::vector<Entry> list;
    std::vector<int> owner;     // relation index (bit - 1) -> entry position, -1 if none
    std::vector<int> of_to;     // target index -> entry position, -1 if none
    std::vector<char> single;   // entry position -> holds exactly one relation
    Remap(const std::vector<Entry> &l, int n_from) : list(l), owner(n_from, -1), single(l.size(), 0) {
        int max_to = -1;
        for (size_t k = 0; k < list.size(); k++) {
            int cnt = 0;
            list[k].from.for_each([&](int b) {
                cnt++;
                if (b - 1 < n_from) owner[b - 1] = (int)k;
            });
            single[k] = cnt == 1;
            max_to = std::max(max_to, list[k].to);
        }
        of_to.assign(max_to + 1, -1);
        for (size_t k = 0; k < list.size(); k++) of_to[list[k].to] = (int)k;
    }
    // remapRelid (:49-59)
    BB rel(const BB &id) const {
        BB out;
        id.for_each([&](int b) {
            int k = (b - 1 < (int)owner.size()) ? owner[b - 1] : -1;
            if (k >= 0) out.set(list[k].to + 1);
        });
        return out;
    }
    // remapRelidNoComposite (:61-75)
    BB rel_nocomp(const BB &id, const GInfo &from) const {
        BB out;
        id.for_each([&](int b) {
            int k = (b - 1 < (int)owner.size()) ? owner[b - 1] : -1;
            if (k < 0) return;
            const Entry &e = list[k];
            if (e.from.size() > 1 || from.base[e.from.lowest_pos() - 1].composite) return;
            out.set(e.to + 1);
        });
        return out;
    }
    // remapRelidInv (:77-87)
    BB inv(const BB &id) const {
        BB out;
        id.for_each([&](int b) {
            int t = b - 1;
            if (t < (int)of_to.size() && of_to[t] >= 0) out |= list[of_to[t]].from;
        });
        return out;
    }
    // Classes whose members fall into fewer than two entries: with entries
    // covering every relation these are the reference's dropped classes (a
    // subset of one entry, countEqClasses :19-47); for a sub-problem's remap
    // they also include classes left with 0 or 1 member, which can never
    // match a join pair.  Either way they are not needed downstream.
    bool ec_below_two_entries(const GInfo &g, int e) const {
        int k0 = -1;
        for (int m : g.ec_members[e]) {
            int k = owner[m];
            if (k < 0) continue;
            if (k0 < 0) k0 = k;
            else if (k != k0) return false;
        }
        return true;
    }

    // remapPlannerInfo (:201-277) with remapEdgeTable / remapBaseRels /
    // remapEqClass (:89-199)
    GInfo info(const GInfo &from) const {
        GInfo to;
        to.n = (int)list.size();
        to.p = from.p;
        to.base.resize(to.n);
        to.edge.assign(to.n, BB());
        for (const Entry &e : list) {
            BB et;
            e.from.for_each([&](int b) { et |= rel(from.edge[b - 1]); });
            et.unset(e.to + 1);
            to.edge[e.to] = et;
            GBase &tb = to.base[e.to];
            tb.id = rel(e.from);
            if (e.qt) {
                tb.rows = e.qt->rows;
                tb.cost = e.qt->cost;
                tb.width = e.qt->width;
                tb.tuples = e.qt->rows;
            } else {
                const GBase &fb = from.base[e.from.lowest_pos() - 1];
                tb.rows = fb.rows;
                tb.cost = fb.cost;
                tb.width = fb.width;
                tb.tuples = fb.tuples;
            }
            tb.composite = (e.from.size() == 1) ? from.base[e.from.lowest_pos() - 1].composite : true;
        }
        // A class with members in two entries contains a listed relation, so
        // a sub-problem (a few relations of a large query) visits only the
        // classes of its relations, in increasing class order like the full
        // scan; the classes it skips are the ones the full scan drops.
        std::vector<int> cand;
        size_t incident = 0;
        for (const Entry &e : list)
            e.from.for_each([&](int b) {
                if (b - 1 < (int)from.rel_ecs.size()) incident += from.rel_ecs[b - 1].size();
            });
        const bool sparse = incident < from.ec.size();
        if (sparse) {
            cand.reserve(incident);
            for (const Entry &e : list)
                e.from.for_each([&](int b) {
                    if (b - 1 < (int)from.rel_ecs.size())
                        cand.insert(cand.end(), from.rel_ecs[b - 1].begin(), from.rel_ecs[b - 1].end());
                });
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        }
        const size_t n_visit = sparse ? cand.size() : from.ec.size();
        if (!sparse) {
            to.ec.reserve(from.ec.size());
            to.sels.reserve(from.sels.size());
            to.fks.reserve(from.fks.size());
            to.vars.reserve(from.vars.size());
        }
        std::vector<int> to_bits;
        for (size_t v = 0; v < n_visit; v++) {
            const size_t i = sparse ? (size_t)cand[v] : v;
            if (ec_below_two_entries(from, (int)i)) continue;
            int s_from = (int)from.ec_members[i].size();
            if (s_from == 2) {
                // both members in single-relation entries (distinct, as the
                // class is not below two entries): the new class has the two
                // targets, member 0 the one with the lower target; the steps
                // below then read sels[0] (ec_index(0, 1, 2) = 0) and each
                // member's own FK mask and column
                const int mm[2] = {from.ec_members[i].begin()[0], from.ec_members[i].begin()[1]};
                const int k0 = owner[mm[0]], k1 = owner[mm[1]];
                if (single[k0] && single[k1]) {
                    BB ect;
                    ect.set(list[k0].to + 1);
                    ect.set(list[k1].to + 1);
                    to.sels.push_back(from.sels[from.ec_off_sels[i]]);
                    const int first = list[k0].to < list[k1].to ? 0 : 1;   // class position of new member 0
                    for (int lt = 0; lt < 2; lt++) {
                        const int lf = lt == 0 ? first : 1 - first;
                        const int rel_f = mm[lf];
                        to.fks.push_back(from.base[rel_f].composite ? BB()
                                                                    : rel_nocomp(from.fks[from.ec_off_fks[i] + lf], from));
                        to.vars.push_back(from.vars[from.ec_off_fks[i] + lf]);
                    }
                    to.ec.push_back(ect);
                    continue;
                }
            }
            const BB &ecf = from.ec[i];
            BB ect = rel(ecf);
            int s_to = ect.size();
            size_t sel_base = to.sels.size(), fk_base = to.fks.size();
            to.sels.resize(sel_base + s_to * (s_to - 1) / 2, 0.0f);
            to.fks.resize(fk_base + s_to, BB());
            to.vars.resize(fk_base + s_to);
            to_bits.clear();
            ect.for_each([&](int b) { to_bits.push_back(b); });
            for (int lt = 0; lt < s_to; lt++) {
                BB id_lt = BB::bit(to_bits[lt]);
                BB id_lf = inv(id_lt);
                int lf = (id_lf.all_lower() & ecf).size();
                for (int rt = lt + 1; rt < s_to; rt++) {
                    BB id_rt = BB::bit(to_bits[rt]);
                    BB id_rf = inv(id_rt);
                    int rf = (id_rf.all_lower() & ecf).size();
                    float v;
                    if (id_lf.size() == 1 && id_rf.size() == 1)
                        v = from.sels[from.ec_off_sels[i] + ec_index(lf, rf, s_from)];
                    else
                        v = estimate_ec_selectivity(from, (int)i, id_lf, id_rf);
                    to.sels[sel_base + ec_index(lt, rt, s_to)] = v;
                }
                if (id_lf.size() == 1 && !from.base[id_lf.lowest_pos() - 1].composite)
                    to.fks[fk_base + lt] = rel_nocomp(from.fks[from.ec_off_fks[i] + lf], from);
                to.vars[fk_base + lt] = from.vars[from.ec_off_fks[i] + lf];
                if (id_lf.size() > 1) to.vars[fk_base + lt].index.available = false;
            }
            to.ec.push_back(ect);
        }
        to.index();
        return to;
    }

    // remapQueryTree (:279-300)
    QT *tree_back(const QT *qt, Arena &A) const {
        if (!qt) return nullptr;
        if (qt->id.size() == 1) {
            int idx = qt->id.lowest_pos() - 1;
            if (idx < (int)of_to.size() && of_to[idx] >= 0 && list[of_to[idx]].qt) return list[of_to[idx]].qt;
        }
        QT *o = A.make();
        o->left = tree_back(qt->left, A);
        o->right = tree_back(qt->right, A);
        // inv distributes over union: an internal node's set is its children's
        if (o->left && o->right && (qt->left->id | qt->right->id) == qt->id) o->id = o->left->id | o->right->id;
        else o->id = inv(qt->id);
        o->rows = qt->rows;
        o->cost = qt->cost;
        o->width = qt->width;
        return o;
    }

    // remapQueryTreeFwd (:302-321)
    QT *tree_fwd(const QT *qt, Arena &A) const {
        if (!qt) return nullptr;
        QT *o = A.make();
        // rel distributes over union: an internal node's set is its children's
        QT *l = nullptr, *r = nullptr;
        if (qt->left && qt->right && (qt->left->id | qt->right->id) == qt->id) {
            l = tree_fwd(qt->left, A);
            r = tree_fwd(qt->right, A);
            o->id = l->id | r->id;
        } else {
            o->id = rel(qt->id);
            if (o->id.size() != 1) {
                l = tree_fwd(qt->left, A);
                r = tree_fwd(qt->right, A);
            }
        }
        if (o->id.size() == 1) {
            o->left = o->right = nullptr;
        } else {
            o->left = l;
            o->right = r;
        }
        o->rows = qt->rows;
        o->cost = qt->cost;
        o->width = qt->width;
        return o;
    }
};

static std::vector<Entry> identity_list(const GInfo &g) {
    std::vector<Entry> l;
    for (int i = 0; i < g.n; i++) l.push_back(Entry{g.base[i].id, i, nullptr});
    return l;
}

// makeBFSIndexRemapper (gpuqo_bfs_indexing.cu:14-55)
static std::vector<Entry> bfs_list(const GInfo &g) {
    std::vector<int> queue(1, 0);
    size_t front = 0;
    std::vector<Entry> l;
    BB seen = BB::bit(1);
    int bfs_idx = 0;
    while (front < queue.size() && bfs_idx < g.n) {
        int b = queue[front++];
        l.push_back(Entry{BB::bit(b + 1), bfs_idx++, nullptr});
        g.edge[b].for_each([&](int next) {
            if (!seen.test(next)) queue.push_back(next - 1);
        });
        seen |= g.edge[b];
    }
    return l;
}

// ---------------------------------------------------------------------------
// exact DP of a remapped sub-problem on the GPU
// ---------------------------------------------------------------------------
static int to_host_info(const GInfo &g, HostInfo &h, std::string &err) {
    if (g.n > 63) {
        err = "sub-problem of " + std::to_string(g.n) + " relations";
        return GPUQO_B200_ERR_TOO_LARGE;
    }
    auto m64 = [](const BB &b) { return b.w[0]; };
    h.n = g.n;
    h.p = g.p;
    h.base.resize(g.n);
    h.edge.resize(g.n);
    for (int i = 0; i < g.n; i++) {
        h.edge[i] = m64(g.edge[i]);
        h.base[i].id = m64(g.base[i].id);
        h.base[i].rows = g.base[i].rows;
        h.base[i].tuples = g.base[i].tuples;
        h.base[i].width = g.base[i].width;
        h.base[i].cost = g.base[i].cost;
        h.base[i].composite = g.base[i].composite;
    }
    // Classes with fewer than two members after remapping (the remapper keeps
    // them, emptied) never match a join pair - they contribute a factor 1 to
    // the selectivity, no quals, no bucket or index candidates - so the DP
    // gets only the classes that can match; its results are unchanged.
    h.ec_relids.clear();
    h.ec_sels.clear();
    h.ec_fks.clear();
    h.ec_vars.clear();
    for (size_t e = 0; e < g.ec.size(); e++) {
        const int s = (int)g.ec_members[e].size();
        if (s < 2) continue;
        h.ec_relids.push_back(m64(g.ec[e]));
        for (int j = 0; j < s * (s - 1) / 2; j++) h.ec_sels.push_back(g.sels[g.ec_off_sels[e] + j]);
        for (int j = 0; j < s; j++) {
            h.ec_fks.push_back(m64(g.fks[g.ec_off_fks[e] + j]));
            h.ec_vars.push_back(g.vars[g.ec_off_fks[e] + j]);
        }
    }
    return 0;
}

struct Ctx {
    DpMode mode;
    Arena A;
    int err = 0;
    std::string msg;
    SubSolver solve;        // exact DP of one remapped sub-problem
    std::atomic<bool> cancel{false};   // this request's own cancel (planner_cancel)

    // InterruptPending (the backend's cancel) or this request's cancel
    bool cancelled() const { return InterruptPending || cancel.load(std::memory_order_relaxed); }
};

static QT *nodes_to_qt(const std::vector<TreeNode> &nodes, int idx, Arena &A) {
    if (idx < 0) return nullptr;
    const TreeNode &t = nodes[idx];
    QT *q = A.make();
    for (uint64_t x = t.set; x; x &= x - 1ull) q->id.set(__builtin_ctzll(x) + 1);
    q->rows = t.rows;
    q->cost.startup = t.startup;
    q->cost.total = t.total;
    q->width = t.width;
    q->left = nodes_to_qt(nodes, t.left, A);
    q->right = nodes_to_qt(nodes, t.right, A);
    return q;
}

// gpuqo_run_idp2_dp (gpuqo_idp.cu:123-141) / gpuqo_run_dpdp_union_dp
// (gpuqo_dpdp_union.cu:254-272): remap, solve, map the plan back
static QT *solve_sub(const GInfo &info, const std::vector<Entry> &list, Ctx &C) {
    // a cancel request ends the IDP loop before its next DP; the drivers
    // unwind normally and the entry point returns NULL with
    // GPUQO_B200_ERR_CANCELLED (the caller's CHECK_FOR_INTERRUPTS then acts)
    if (C.cancelled()) {
        C.err = GPUQO_B200_ERR_CANCELLED;
        C.msg = "cancelled between IDP iterations";
        return nullptr;
    }
    Remap R(list, info.n);
    GInfo sub = R.info(info);
    HostInfo h;
    if (int rc = to_host_info(sub, h, C.msg)) {
        C.err = rc;
        return nullptr;
    }
    std::vector<TreeNode> nodes;
    int rc = C.solve ? C.solve(h, C.mode, nodes, C.msg) : exact_dp(h, C.mode, nodes, C.msg);
    if (rc) {
        C.err = rc;
        return nullptr;
    }
    QT *qt = nodes_to_qt(nodes, 0, C.A);
    return R.tree_back(qt, C.A);
}

// ---------------------------------------------------------------------------
// GOO (gpuqo_cpu_goo.cu:61-150): greedy on the smallest intermediate result
// ---------------------------------------------------------------------------
struct GooNode {
    QT *qt;
    BB edges;      // union of the relations' edges (are_connected_ids operand)
};

static QT *goo(const GInfo &g, Arena &A) {
    auto compare = [](QT *l, QT *r) {
        if (l != nullptr && r != nullptr) return l->rows > r->rows;
        return r != nullptr;
    };
    std::vector<QT *> heap;
    std::map<BB, GooNode> rels;
    auto edges_of = [&](const BB &id) {
        BB e;
        id.for_each([&](int b) { e |= g.edge[b - 1]; });
        return e;
    };
    auto join = [&](QT &l, QT &r) {
        QT *q = A.make();
        q->id = l.id | r.id;
        q->rows = estimate_join_rows(g, l, r);
        q->cost.startup = 0;
        q->cost.total = q->rows + l.cost.total + r.cost.total;
        q->left = &l;
        q->right = &r;
        q->width = l.width + r.width;
        return q;
    };
    for (int i = 0; i < g.n; i++) {
        QT *q = A.make();
        q->id = g.base[i].id;
        q->rows = g.base[i].rows;
        q->cost.startup = 0;
        q->cost.total = g.base[i].rows;
        q->width = g.base[i].width;
        rels.emplace(q->id, GooNode{q, edges_of(q->id)});
    }
    // are_valid_pair (gpuqo_filter.cuh:84-90): connected and disjoint.  The
    // reference tests every pair of entries in map order; the entries valid
    // with `a` are those holding a relation of a's edges outside a, so they
    // are found through owner[] (relation -> its entry) and visited in the
    // same map order, which keeps the heap's push sequence and so its ties.
    using It = std::map<BB, GooNode>::iterator;
    std::vector<It> owner(g.n + 1, rels.end());
    for (It it = rels.begin(); it != rels.end(); ++it)
        it->first.for_each([&](int b) {
            if (b <= g.n) owner[b] = it;
        });
    std::vector<It> cand;
    auto valid_entries = [&](const GooNode &a) {
        cand.clear();
        (a.edges - a.qt->id).for_each([&](int b) {
            if (b <= g.n && owner[b] != rels.end()) cand.push_back(owner[b]);
        });
        std::sort(cand.begin(), cand.end(), [](const It &x, const It &y) { return x->first < y->first; });
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    };
    for (It i = rels.begin(); i != rels.end(); ++i) {
        valid_entries(i->second);
        for (const It &j : cand)
            if (i->first < j->first) {
                heap.push_back(join(*i->second.qt, *j->second.qt));
                std::push_heap(heap.begin(), heap.end(), compare);
            }
    }
    QT *smallest = nullptr;
    do {
        if (heap.empty()) return nullptr;   // disconnected query graph
        std::pop_heap(heap.begin(), heap.end(), compare);
        smallest = heap.back();
        heap.pop_back();
        auto lp = rels.find(smallest->left->id);
        auto rp = rels.find(smallest->right->id);
        if (lp == rels.end() || rp == rels.end()) {
            smallest = nullptr;
            continue;
        }
        // edges_of distributes over the union of the two entries
        GooNode sn{smallest, lp->second.edges | rp->second.edges};
        rels.erase(lp);
        rels.erase(rp);
        valid_entries(sn);
        for (const It &j : cand) {
            heap.push_back(join(*smallest, *j->second.qt));
            std::push_heap(heap.begin(), heap.end(), compare);
        }
        const It ins = rels.emplace(smallest->id, sn).first;
        smallest->id.for_each([&](int b) {
            if (b <= g.n) owner[b] = ins;
        });
    } while (smallest == nullptr || smallest->id.size() < g.n);
    return smallest;
}

// ---------------------------------------------------------------------------
// IDP2 (gpuqo_idp.cu:96-297)
// ---------------------------------------------------------------------------
static QT *most_expensive_subtree(QT *qt, int max_size) {
    if (qt->id.size() <= max_size) return qt;
    QT *l = most_expensive_subtree(qt->left, max_size);
    QT *r = most_expensive_subtree(qt->right, max_size);
    if (l->id.size() == 1) return r;
    if (r->id.size() == 1) return l;
    if (l->cost.total > r->cost.total) return l;
    if (l->cost.total < r->cost.total) return r;
    if (l->id.size() < r->id.size()) return l;
    return r;
}

static QT *idp2_rec(QT *goo_qt, const GInfo &info, const std::vector<Entry> &list, int n_iters, Ctx &C) {
    Remap R(list, info.n);
    GInfo ni = R.info(info);
    QT *ngoo = R.tree_fwd(goo_qt, C.A);
    const int iters = std::min(ni.n, n_iters);
    QT *maximal = most_expensive_subtree(ngoo, iters);
    std::vector<Entry> reopt;
    {
        int i = 0;
        maximal->id.for_each([&](int b) { reopt.push_back(Entry{BB::bit(b), i++, nullptr}); });
    }
    QT *reopt_qt = solve_sub(ni, reopt, C);
    if (!reopt_qt) return nullptr;
    QT *res;
    if (iters == ni.n) {
        res = reopt_qt;
    } else {
        std::vector<Entry> next;
        next.push_back(Entry{reopt_qt->id, 0, reopt_qt});
        int j = 1;
        for (int i = 0; i < ni.n; i++)
            if (!ni.base[i].id.is_subset_of(reopt_qt->id)) next.push_back(Entry{ni.base[i].id, j++, nullptr});
        res = idp2_rec(ngoo, ni, next, n_iters, C);
        if (!res) return nullptr;
    }
    return R.tree_back(res, C.A);
}

static QT *run_idp2(const GInfo &info, int n_iters, Ctx &C) {
    QT *goo_qt = goo(info, C.A);
    if (!goo_qt) {
        C.err = GPUQO_B200_ERR_ARGS;
        C.msg = "query graph is not connected";
        return nullptr;
    }
    return idp2_rec(goo_qt, info, identity_list(info), n_iters, C);
}

// ---------------------------------------------------------------------------
// UnionDP (gpuqo_dpdp_union.cu:29-472)
// ---------------------------------------------------------------------------
struct GraphEdge {
    BB left, right;
    int left_size, right_size, total_size;
    float rows, selectivity, weight;
};

struct CompareEdges {
    bool operator()(const GraphEdge *l, const GraphEdge *r) const {
        if (l->total_size == r->total_size) return l->weight > r->weight;
        return l->total_size > r->total_size;
    }
};

static QT *union_rec(const GInfo &info, const std::vector<Entry> &list, int n_iters, Ctx &C) {
    Remap R(list, info.n);
    GInfo ni = R.info(info);
    const int iters = std::min(ni.n, n_iters);
    if (ni.n == iters) return solve_sub(info, list, C);

    // fillPriorityQueues (:212-251): edges in the reference's BFS order,
    // weight = selectivity * rows * rows (createGraphEdge :164-209)
    std::vector<std::unique_ptr<GraphEdge>> edges;
    std::priority_queue<GraphEdge *, std::vector<GraphEdge *>, CompareEdges> pq;
    {
        std::queue<int> bq;
        int bfs_idx = 0;
        bq.push(0);
        BB seen2 = BB::bit(1);
        while (!bq.empty() && bfs_idx < ni.n) {
            int b = bq.front();
            bq.pop();
            bfs_idx++;
            ni.edge[b].for_each([&](int next) {
                if (seen2.test(next)) return;
                bq.push(next - 1);
                GraphEdge *e = new GraphEdge();
                e->left = ni.base[b].id;
                e->right = ni.base[next - 1].id;
                e->selectivity = estimate_join_selectivity(ni, e->left, e->right);
                e->rows = e->selectivity * ni.base[b].rows * ni.base[next - 1].rows;
                e->left_size = e->right_size = 1;
                e->total_size = 2;
                e->weight = e->rows;
                edges.emplace_back(e);
                pq.push(e);
            });
            seen2 |= BB::bit(b + 1);
        }
    }
    // DisjointSet over relation indices (:36-101)
    std::vector<int> parent(ni.n), size(ni.n, 1);
    std::vector<BB> csg(ni.n);
    for (int i = 0; i < ni.n; i++) {
        parent[i] = i;
        csg[i] = ni.base[i].id;
    }
    std::function<int(int)> find = [&](int x) {
        if (parent[x] != x) parent[x] = find(parent[x]);
        return parent[x];
    };
    const int upper_threshold = 16;
    while (!pq.empty()) {
        GraphEdge *e = pq.top();
        pq.pop();
        int l = e->left.lowest_pos() - 1, r = e->right.lowest_pos() - 1;
        int x = find(l), y = find(r);
        if (x == y) continue;
        if (e->total_size != size[x] + size[y]) {
            e->left_size = size[x];
            e->right_size = size[y];
            e->total_size = e->left_size + e->right_size;
            pq.push(e);
        } else if (e->total_size < upper_threshold) {
            if (size[x] > size[y]) {
                parent[y] = x;
                size[x] += size[y];
                csg[x] |= csg[y];
            } else if (size[x] < size[y]) {
                parent[x] = y;
                size[y] += size[x];
                csg[y] |= csg[x];
            } else {
                parent[x] = y;
                size[y] *= 2;
                csg[y] |= csg[x];
            }
        }
    }
    std::vector<BB> subgraphs;
    BB seen;
    for (int i = 0; i < ni.n; i++) {
        const BB &cs = csg[find(i)];
        if (!cs.is_subset_of(seen)) subgraphs.push_back(cs);
        seen |= cs;
    }
    std::vector<Entry> next;
    for (size_t i = 0; i < subgraphs.size(); i++) {
        std::vector<Entry> reopt;
        int j = 0;
        subgraphs[i].for_each([&](int b) { reopt.push_back(Entry{BB::bit(b), j++, nullptr}); });
        QT *q = solve_sub(ni, reopt, C);
        if (!q) return nullptr;
        next.push_back(Entry{q->id, (int)i, q});
    }
    QT *res = union_rec(ni, next, n_iters, C);
    if (!res) return nullptr;
    return R.tree_back(res, C.A);
}

// ---------------------------------------------------------------------------
// entry
// ---------------------------------------------------------------------------
static QueryTreeC *qt_to_c(const QT *q) {
    if (!q) return nullptr;
    QueryTreeC *o = (QueryTreeC *)palloc(sizeof(QueryTreeC));
    int top = 0;
    for (int i = 0; i < kBigWords; i++)
        if (q->id.w[i]) top = i;
    int nwords = top + 1;
    Bitmapset *b = (Bitmapset *)palloc0(offsetof(Bitmapset, words) + nwords * sizeof(bitmapword));
    b->nwords = nwords;
    for (int i = 0; i < nwords; i++) b->words[i] = q->id.w[i];
    o->id = b;
    o->rows = q->rows;
    o->cost = q->cost;
    o->width = q->width;
    o->left = qt_to_c(q->left);
    o->right = qt_to_c(q->right);
    return o;
}

// One planning request (__gpuqo_run, gpuqo_main_internal.cu:82-160): BFS
// relabel, IDP2 / UnionDP or one exact DP, plan mapped back to the caller's
// numbering.  Settings are captured by the caller (no GUC reads here).
struct Planner {
    Ctx C;
    GInfo g;
    int idp_n_iters = 0, idp_type = GPUQO_IDP2;
    bool spanning = false;   // gpuqo_spanning_tree_enable at creation
    QT *result = nullptr;

    int run() {
        if (spanning) spanning_tree(g);
        std::vector<Entry> bl = bfs_list(g);
        if ((int)bl.size() != g.n) {
            C.msg = "query graph is not connected";
            return GPUQO_B200_ERR_ARGS;
        }
        Remap R(bl, g.n);
        GInfo rg = R.info(g);
        const bool idp = idp_n_iters > 1 && idp_n_iters < g.n;
        QT *qt = nullptr;
        if (idp) {
            if (idp_type == GPUQO_IDP2) qt = run_idp2(rg, idp_n_iters, C);
            else if (idp_type == GPUQO_UNION) qt = union_rec(rg, identity_list(rg), idp_n_iters, C);
            else {
                C.msg = "gpuqo_idp_type: only IDP2 and UNION are provided";
                return GPUQO_B200_ERR_UNSUPPORTED;
            }
        } else if (g.n <= 63) {
            if (C.cancelled()) {
                C.msg = "cancelled before the exact DP";
                return GPUQO_B200_ERR_CANCELLED;
            }
            HostInfo h;
            if (int rc = to_host_info(rg, h, C.msg)) return rc;
            std::vector<TreeNode> nodes;
            int rc = C.solve ? C.solve(h, C.mode, nodes, C.msg) : exact_dp(h, C.mode, nodes, C.msg);
            if (rc) return rc;
            qt = nodes_to_qt(nodes, 0, C.A);
        } else {
            C.msg = std::to_string(g.n) + " relations need IDP (set gpuqo_idp_n_iters between 2 and n-1)";
            return GPUQO_B200_ERR_UNSUPPORTED;
        }
        if (!qt) return C.err ? C.err : GPUQO_B200_ERR_ARGS;
        result = R.tree_back(qt, C.A);
        return 0;
    }
};

PlannerHandle *planner_new(int algorithm, const GpuqoPlannerInfoC *info_c, int idp_n_iters, int idp_type,
                           SubSolver solver, std::string &err) {
    Planner *p = new Planner();
    if (!convert_big(info_c, p->g, err)) {
        delete p;
        return nullptr;
    }
    p->C.mode = mode_for(algorithm);
    p->C.solve = std::move(solver);
    p->idp_n_iters = idp_n_iters;
    p->idp_type = idp_type;
    p->spanning = gpuqo_spanning_tree_enable;
    return reinterpret_cast<PlannerHandle *>(p);
}

void planner_cancel(PlannerHandle *h) {
    reinterpret_cast<Planner *>(h)->C.cancel.store(true, std::memory_order_relaxed);
}

int planner_run(PlannerHandle *h, std::string &err) {
    Planner *p = reinterpret_cast<Planner *>(h);
    int rc = p->run();
    if (rc) err = p->C.msg.empty() ? "planning failed" : p->C.msg;
    return rc;
}

QueryTreeC *planner_result(PlannerHandle *h) { return qt_to_c(reinterpret_cast<Planner *>(h)->result); }

void planner_free(PlannerHandle *h) { delete reinterpret_cast<Planner *>(h); }

QueryTreeC *run_planned(int algorithm, GpuqoPlannerInfoC *info_c) {
    std::string err;
    const int n = info_c->n_rels;
    const bool idp = gpuqo_idp_n_iters > 1 && gpuqo_idp_n_iters < n;
    if (!idp && n > 63) {
        set_error(GPUQO_B200_ERR_UNSUPPORTED,
                  std::to_string(n) + " relations need IDP (set gpuqo_idp_n_iters between 2 and n-1)");
        return nullptr;
    }
    if (idp && gpuqo_idp_type != GPUQO_IDP2 && gpuqo_idp_type != GPUQO_UNION) {
        set_error(GPUQO_B200_ERR_UNSUPPORTED, "gpuqo_idp_type: only IDP2 and UNION are provided");
        return nullptr;
    }
    PlannerHandle *h = planner_new(algorithm, info_c, gpuqo_idp_n_iters, gpuqo_idp_type, nullptr, err);
    if (!h) {
        set_error(GPUQO_B200_ERR_ARGS, err);
        return nullptr;
    }
    int rc = planner_run(h, err);
    QueryTreeC *out = rc ? nullptr : planner_result(h);
    planner_free(h);
    if (rc) set_error(rc, err);
    return out;
}

}  // namespace gqb
