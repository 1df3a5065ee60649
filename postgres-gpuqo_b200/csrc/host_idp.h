// host_idp.h - IDP2 / UnionDP drivers over the GPU exact DP.
#pragma once

#include <string>

#include "gpuqo_b200.h"

namespace gqb {

// Entry used by gpuqo_run when 1 < gpuqo_idp_n_iters < n_rels, or when the
// query has 64 or more relations.
QueryTreeC *run_idp(int algorithm, GpuqoPlannerInfoC *info);

void set_error(int code, const std::string &msg);

}  // namespace gqb
