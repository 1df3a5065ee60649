// host_info.h - host-side planner info (after conversion from the C ABI),
// its BFS relabelling, and the device blob built from it.
//
// Masks use the reference's Postgres layout: relation i is bit i+1.  A
// HostInfo holds up to 63 relations in 64-bit masks (the reference's
// Bitmapset32 / Bitmapset64 cases, gpuqo_main_internal.cu:178-181); larger
// queries go through the IDP drivers on dynamic bitsets (host_idp.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dp_engine.h"
#include "gpuqo_b200.h"

namespace gqb {

typedef uint64_t mask64;

struct HostParams {
    // GpuqoPlannerInfoParams (gpuqo_planner_info.cuh:90-107), filled by
    // setParams (gpuqo_planner_info.cu:114-131): doubles narrowed to float.
    float effective_cache_size, seq_page_cost, random_page_cost, cpu_tuple_cost, cpu_index_tuple_cost,
        cpu_operator_cost, disable_cost;
    bool enable_seqscan, enable_indexscan, enable_tidscan, enable_sort, enable_hashagg, enable_nestloop,
        enable_mergejoin, enable_hashjoin;
    int work_mem;
};

struct HostBaseRel {
    mask64 id;
    float rows, tuples;
    int width;
    PathCost cost;
    bool composite;
};

struct HostInfo {
    int n = 0;
    HostParams p;
    std::vector<HostBaseRel> base;     // [n]
    std::vector<mask64> edge;          // [n]
    std::vector<mask64> ec_relids;     // [n_ec]
    std::vector<float> ec_sels;
    std::vector<mask64> ec_fks;
    std::vector<VarInfo> ec_vars;
};

// Reads the Postgres cost GUCs the way setParams does.
HostParams read_params();

// GpuqoPlannerInfoC -> HostInfo (gpuqo_planner_info.cu:134-200); n_rels < 64.
bool convert_info(const GpuqoPlannerInfoC *c, HostInfo &out, std::string &err);

// BFS order of makeBFSIndexRemapper (gpuqo_bfs_indexing.cu:14-55):
// from_of_to[t] = original relation index placed at position t.
std::vector<int> bfs_order(const HostInfo &info);

// Relabels single relations (remapPlannerInfo for a list of single-relation
// entries, gpuqo_remapper.cu:201-277).
HostInfo relabel(const HostInfo &from, const std::vector<int> &from_of_to);

// Device planner-info blob (compact masks, bit i = relation i); n <= 32.
std::vector<uint32_t> build_blob(const HostInfo &info);

// Plain DPsub with gpuqo_dpsub_csg_enable on a graph with fewer than half of
// all possible edges: the DP runs on the block (MPDP) enumeration, which
// visits only the valid csg-cmp pairs, with candidates keyed by their
// plain-DPsub index (DevHeader::index_order), so the plan is cpu_dpsub's.
// Switches mode to kModeMpdp and marks the blob; no change otherwise.
void apply_dpsub_csg(std::vector<uint32_t> &blob, DpMode &mode);

}  // namespace gqb
