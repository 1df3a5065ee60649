/*
 * Host-side stubs that let the reference's gpuqo sources link into a
 * standalone shared library (oracle/_ref/libgpuqo_ref.so) outside Postgres.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle ("reference
 * run here"): tests, the smoke check and bench.py's CPU-baseline leg may load
 * it as a checker; the product library never links or calls it.
 *
 * What the gpuqo module expects from the Postgres backend, and what is
 * supplied here instead:
 *   - palloc/palloc0/pfree (src/backend/optimizer/gpuqo/gpuqo_postgres.cuh:15-16;
 *     gpuqo_planner_info.cu:259 allocates the returned QueryTreeC with palloc)
 *     -> malloc/calloc/free.
 *   - InterruptPending / ProcessInterrupts (gpuqo.cuh:20-28) -> a flag that
 *     stays 0 and a no-op.
 *   - the Postgres cost GUCs read by setParams (gpuqo_planner_info.cu:84-131)
 *     -> Postgres 12 defaults, with the enable_* flags set as the reference's
 *     README "Limitations" section prescribes.
 *   - gpuqo_algorithm (defined in gpuqo_main.c:43, which is not compiled here).
 *   - bms_* (nodes/bitmapset.c) for BitmapsetDynamic (>= 64 relations) ->
 *     small re-implementations with Postgres 12 semantics (empty sets may be
 *     NULL; sets are never shrunk).
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <csignal>
#include <cstdio>
#include <cstddef>

typedef uint64_t bitmapword;
#define BITS_PER_BITMAPWORD 64

struct Bitmapset {
    int nwords;
    bitmapword words[1];
};

extern "C" {

void *palloc(size_t size) { return malloc(size ? size : 1); }
void *palloc0(size_t size) { return calloc(1, size ? size : 1); }
void pfree(void *p) { free(p); }

volatile sig_atomic_t InterruptPending = 0;
void ProcessInterrupts(void) {}

/* Postgres cost GUCs (src/backend/optimizer/path/costsize.c defaults). */
double seq_page_cost = 1.0;
double random_page_cost = 4.0;
double cpu_tuple_cost = 0.01;
double cpu_index_tuple_cost = 0.005;
double cpu_operator_cost = 0.0025;
double parallel_tuple_cost = 0.1;
double parallel_setup_cost = 1000.0;
int effective_cache_size = 524288;
double disable_cost = 1.0e10;
int max_parallel_workers_per_gather = 2;
bool enable_seqscan = true;
bool enable_indexscan = true;
bool enable_indexonlyscan = false;
bool enable_bitmapscan = false;
bool enable_tidscan = false;
bool enable_sort = true;
bool enable_hashagg = true;
bool enable_nestloop = true;
bool enable_material = false;
bool enable_mergejoin = false;
bool enable_hashjoin = true;
bool enable_gathermerge = false;
bool enable_partitionwise_join = false;
bool enable_partitionwise_aggregate = false;
bool enable_parallel_append = true;
bool enable_parallel_hash = false;
bool enable_partition_pruning = true;
int work_mem = 4096;

int gpuqo_algorithm = 0;

/* ---------------- bitmapset (Postgres 12 semantics) ---------------- */

static size_t bms_bytes(int nwords) {
    return offsetof(Bitmapset, words) + (size_t)nwords * sizeof(bitmapword);
}

static Bitmapset *bms_alloc(int nwords) {
    Bitmapset *r = (Bitmapset *)palloc0(bms_bytes(nwords));
    r->nwords = nwords;
    return r;
}

Bitmapset *bms_copy(const Bitmapset *a) {
    if (a == NULL) return NULL;
    Bitmapset *r = (Bitmapset *)palloc(bms_bytes(a->nwords));
    memcpy(r, a, bms_bytes(a->nwords));
    return r;
}

bool bms_equal(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) {
        if (b == NULL) return true;
        for (int i = 0; i < b->nwords; i++) if (b->words[i]) return false;
        return true;
    }
    if (b == NULL) {
        for (int i = 0; i < a->nwords; i++) if (a->words[i]) return false;
        return true;
    }
    const Bitmapset *s = a->nwords <= b->nwords ? a : b;
    const Bitmapset *l = a->nwords <= b->nwords ? b : a;
    int i = 0;
    for (; i < s->nwords; i++) if (s->words[i] != l->words[i]) return false;
    for (; i < l->nwords; i++) if (l->words[i]) return false;
    return true;
}

int bms_compare(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return bms_equal(a, b) ? 0 : -1;
    if (b == NULL) return bms_equal(a, b) ? 0 : +1;
    int shortlen = a->nwords < b->nwords ? a->nwords : b->nwords;
    for (int i = shortlen; i < a->nwords; i++) if (a->words[i]) return +1;
    for (int i = shortlen; i < b->nwords; i++) if (b->words[i]) return -1;
    for (int i = shortlen - 1; i >= 0; i--) {
        if (a->words[i] != b->words[i]) return a->words[i] > b->words[i] ? +1 : -1;
    }
    return 0;
}

Bitmapset *bms_make_singleton(int x) {
    if (x < 0) { fprintf(stderr, "bms_make_singleton: negative member\n"); abort(); }
    Bitmapset *r = bms_alloc(x / BITS_PER_BITMAPWORD + 1);
    r->words[x / BITS_PER_BITMAPWORD] = (bitmapword)1 << (x % BITS_PER_BITMAPWORD);
    return r;
}

void bms_free(Bitmapset *a) { if (a) pfree(a); }

Bitmapset *bms_union(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return bms_copy(b);
    if (b == NULL) return bms_copy(a);
    const Bitmapset *s = a->nwords <= b->nwords ? a : b;
    const Bitmapset *l = a->nwords <= b->nwords ? b : a;
    Bitmapset *r = bms_copy(l);
    for (int i = 0; i < s->nwords; i++) r->words[i] |= s->words[i];
    return r;
}

Bitmapset *bms_intersect(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL || b == NULL) return NULL;
    const Bitmapset *s = a->nwords <= b->nwords ? a : b;
    const Bitmapset *l = a->nwords <= b->nwords ? b : a;
    Bitmapset *r = bms_copy(s);
    for (int i = 0; i < s->nwords; i++) r->words[i] &= l->words[i];
    return r;
}

Bitmapset *bms_difference(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return NULL;
    if (b == NULL) return bms_copy(a);
    Bitmapset *r = bms_copy(a);
    int n = a->nwords < b->nwords ? a->nwords : b->nwords;
    for (int i = 0; i < n; i++) r->words[i] &= ~b->words[i];
    return r;
}

bool bms_is_subset(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return true;
    if (b == NULL) {
        for (int i = 0; i < a->nwords; i++) if (a->words[i]) return false;
        return true;
    }
    int n = a->nwords < b->nwords ? a->nwords : b->nwords;
    for (int i = 0; i < n; i++) if (a->words[i] & ~b->words[i]) return false;
    for (int i = n; i < a->nwords; i++) if (a->words[i]) return false;
    return true;
}

bool bms_is_member(int x, const Bitmapset *a) {
    if (x < 0) { fprintf(stderr, "bms_is_member: negative member\n"); abort(); }
    if (a == NULL) return false;
    int w = x / BITS_PER_BITMAPWORD;
    if (w >= a->nwords) return false;
    return (a->words[w] >> (x % BITS_PER_BITMAPWORD)) & 1;
}

bool bms_overlap(const Bitmapset *a, const Bitmapset *b) {
    if (a == NULL || b == NULL) return false;
    int n = a->nwords < b->nwords ? a->nwords : b->nwords;
    for (int i = 0; i < n; i++) if (a->words[i] & b->words[i]) return true;
    return false;
}

int bms_num_members(const Bitmapset *a) {
    if (a == NULL) return 0;
    int c = 0;
    for (int i = 0; i < a->nwords; i++) c += __builtin_popcountll(a->words[i]);
    return c;
}

bool bms_is_empty(const Bitmapset *a) {
    if (a == NULL) return true;
    for (int i = 0; i < a->nwords; i++) if (a->words[i]) return false;
    return true;
}

Bitmapset *bms_add_member(Bitmapset *a, int x) {
    if (x < 0) { fprintf(stderr, "bms_add_member: negative member\n"); abort(); }
    if (a == NULL) return bms_make_singleton(x);
    int w = x / BITS_PER_BITMAPWORD;
    if (w >= a->nwords) {
        Bitmapset *r = bms_alloc(w + 1);
        memcpy(r->words, a->words, a->nwords * sizeof(bitmapword));
        pfree(a);
        a = r;
    }
    a->words[w] |= (bitmapword)1 << (x % BITS_PER_BITMAPWORD);
    return a;
}

Bitmapset *bms_del_member(Bitmapset *a, int x) {
    if (x < 0) { fprintf(stderr, "bms_del_member: negative member\n"); abort(); }
    if (a == NULL) return NULL;
    int w = x / BITS_PER_BITMAPWORD;
    if (w < a->nwords) a->words[w] &= ~((bitmapword)1 << (x % BITS_PER_BITMAPWORD));
    return a;
}

Bitmapset *bms_add_members(Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return bms_copy(b);
    if (b == NULL) return a;
    if (a->nwords < b->nwords) {
        Bitmapset *r = bms_copy(b);
        for (int i = 0; i < a->nwords; i++) r->words[i] |= a->words[i];
        pfree(a);
        return r;
    }
    for (int i = 0; i < b->nwords; i++) a->words[i] |= b->words[i];
    return a;
}

Bitmapset *bms_add_range(Bitmapset *a, int lower, int upper) {
    for (int x = lower; x <= upper; x++) a = bms_add_member(a, x);
    return a;
}

Bitmapset *bms_int_members(Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return NULL;
    if (b == NULL) { pfree(a); return NULL; }
    int i = 0;
    for (; i < a->nwords && i < b->nwords; i++) a->words[i] &= b->words[i];
    for (; i < a->nwords; i++) a->words[i] = 0;
    return a;
}

Bitmapset *bms_del_members(Bitmapset *a, const Bitmapset *b) {
    if (a == NULL) return NULL;
    if (b == NULL) return a;
    int n = a->nwords < b->nwords ? a->nwords : b->nwords;
    for (int i = 0; i < n; i++) a->words[i] &= ~b->words[i];
    return a;
}

Bitmapset *bms_join(Bitmapset *a, Bitmapset *b) {
    if (a == NULL) return b;
    if (b == NULL) return a;
    Bitmapset *r = bms_add_members(a, b);
    if (r != b) pfree(b);
    return r;
}

uint32_t bms_hash_value(const Bitmapset *a) {
    /* FNV-1a over the non-zero prefix; any consistent hash serves the
     * unordered containers the reference keys by BitmapsetDynamic. */
    if (a == NULL) return 0;
    int last = a->nwords;
    while (last > 0 && a->words[last - 1] == 0) last--;
    uint32_t h = 2166136261u;
    const unsigned char *p = (const unsigned char *)a->words;
    for (size_t i = 0; i < (size_t)last * sizeof(bitmapword); i++) {
        h ^= p[i];
        h *= 16777619u;
    }
    return h;
}

/* ---------------- harness helpers exported to the Python driver ------------ */

struct PathCostRef { float startup; float total; };
struct QueryTreeRef {
    Bitmapset *id;
    float rows;
    PathCostRef cost;
    int width;
    QueryTreeRef *left;
    QueryTreeRef *right;
};

void ref_free_query_tree(QueryTreeRef *qt) {
    if (qt == NULL) return;
    ref_free_query_tree(qt->left);
    ref_free_query_tree(qt->right);
    bms_free(qt->id);
    pfree(qt);
}

}  /* extern "C" */
