// host_idp.h - IDP2 / UnionDP drivers over the GPU exact DP.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "dp_engine.h"
#include "gpuqo_b200.h"
#include "host_info.h"

namespace gqb {

// Exact DP of one (remapped, at most 63-relation) sub-problem.
using SubSolver = std::function<int(const HostInfo &, DpMode, std::vector<TreeNode> &, std::string &)>;

// A planning request: BFS relabel, IDP2 / UnionDP (1 < idp_n_iters < n) or one
// exact DP, with every exact DP done by `solver` (the GPU engine directly when
// empty).  Used by run_idp and by the serving loop.
struct PlannerHandle;
PlannerHandle *planner_new(int algorithm, const GpuqoPlannerInfoC *info, int idp_n_iters, int idp_type,
                           SubSolver solver, std::string &err);
int planner_run(PlannerHandle *p, std::string &err);
// Asks a planner to stop: it returns GPUQO_B200_ERR_CANCELLED before its next
// exact DP (thread-safe; a planner that has finished keeps its result).
void planner_cancel(PlannerHandle *p);
QueryTreeC *planner_result(PlannerHandle *p);   // palloc'd, caller's numbering
void planner_free(PlannerHandle *p);

// Entry used by gpuqo_run when 1 < gpuqo_idp_n_iters < n_rels, when the
// query has 64 or more relations, or when gpuqo_spanning_tree_enable is set:
// the planner on dynamic bitsets (spanning tree, BFS relabel, IDP2 / UnionDP
// or one exact DP of at most 63 relations).
QueryTreeC *run_planned(int algorithm, GpuqoPlannerInfoC *info);

void set_error(int code, const std::string &msg);

}  // namespace gqb
