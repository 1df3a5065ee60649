// dp_engine.h - host interface of the device DP engine (dp_kernels.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dp_layout.h"

namespace gqb {

enum DpMode : int {
    kModeDpsub = 0,   // all-subsets enumeration (gpuqo_algorithm=dpsub, bicc off)
    kModeMpdp = 1,    // biconnected-block enumeration (bicc on)
    kModeDpsize = 2,  // DPsize (gpuqo_algorithm=dpsize): cpu_dpsize's level-list order and ties
};

// One node of the extracted plan, compact masks (bit i = relation i; the
// dense-memo kernels write sets of up to 32 relations, the sparse exact DP of
// 32 to 63 relations the full 64 bits).
struct TreeNode {
    uint64_t set;
    int32_t left, right;          // node indices, -1 for leaves
    float rows, startup, total;
    int32_t width;
};

struct EngineStats {
    uint64_t connected_sets = 0;
    uint64_t evaluated_pairs = 0;
    uint64_t filtered_subsets = 0;
    uint64_t memo_bytes = 0;
    double device_ms = 0.0;
    double eval_kernel_ms = 0.0;
    uint32_t eval_kernel_launches = 0;
    uint32_t kernel_launches = 0;
    uint32_t fallback_sets = 0;
    uint32_t barrier_timeouts = 0;     // persistent launches whose grid barrier gave up (rerun per level)
    double handoff_ms = 0.0;           // device time of the batch's queries run alone (they fill the GPU)
};

// Runs one exact DP on the calling thread's current device.  `blob` is the
// device planner info (DevHeader + class arrays, see dp_device.cuh).  On
// success fills `nodes` (root first) and returns 0; otherwise a
// GPUQO_B200_ERR_* code and a message in `err`.
int engine_run(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, bool profile,
               std::vector<TreeNode> &nodes, EngineStats &stats, std::string &err);

// Device-resident timing of one DP (planner info uploaded once, the DP graph
// replayed `iters` times, CUDA events on the engine stream, optional L2 flush
// between replays).  Also returns the plan of the last replay.
int engine_time_resident(const std::vector<uint32_t> &blob, int n, DpMode mode, bool ccc, int warmup, int iters,
                         bool flush_l2, double &ms_per_iter, std::vector<TreeNode> &nodes, EngineStats &stats,
                         std::string &err);

// Batched MPDP of many sub-problems (each <= 30 relations and eligible, see
// batch_eligible), level-synchronous per wave; waves are consecutive queries
// whose memory stays within wave_bytes.  out[i] gets query i's plan nodes.
int engine_run_batch(const std::vector<const std::vector<uint32_t> *> &blobs, uint64_t wave_bytes,
                     std::vector<std::vector<TreeNode>> &out, EngineStats &stats, std::vector<double> &wave_ms,
                     std::string &err);
bool batch_eligible(const std::vector<uint32_t> &blob);
// Relative work of one exact DP (connected sets times candidates per set, from
// the exact count on tree-shaped graphs, an upper bound otherwise): the
// weight by which a batch is spread over devices.
double engine_work_estimate(const std::vector<uint32_t> &blob);
// Host-side helpers of the multi-device batch and service (host_api.cpp).
void plan_shards(const double *work, int n, int n_dev, int *dev_of);
int batch_devices(std::vector<int> &devs, std::string &err);
uint64_t batch_query_bytes(int n);

// Exact DP of 32 to 63 relations (MPDP, or plain DPsub on its valid pairs)
// with the connected sets enumerated on the host and a device hash-table memo
// (dp_wide.cu); sparse query graphs only (at most wide_set_capacity()
// connected sets, else GPUQO_B200_ERR_TOO_LARGE).
struct HostInfo;
int engine_run_wide(const HostInfo &info, DpMode mode, std::vector<TreeNode> &nodes, EngineStats &st,
                    std::string &err);
uint64_t wide_set_capacity();
// whether an exact DP of n relations in this mode runs on the sparse memo
// (n > 31, or n >= gpuqo_b200_sparse_from_rels for DPsub and MPDP)
bool use_sparse_memo(int n, DpMode mode);

// Device-memory estimate (bytes) of one exact DP over n relations.
uint64_t engine_bytes_needed(int n);

// Measures, on the given tree-shaped blobs (growing sizes), the counts of
// connected sets per level up to which the 2-blocks-per-SM tree kernel wins
// and from which the 4-blocks-per-SM tree kernel wins, the total count from
// which single launches win over batch waves, and installs them for the
// current device.
int engine_autotune(const std::vector<std::vector<uint32_t>> &blobs, double &single_narrow_level_sets,
                    double &single_wide_level_sets, double &batch_single_sets, std::string &err);
// Installs crossovers measured earlier (or the defaults) for the current device.
void engine_set_tuning(double single_narrow_level_sets, double single_wide_level_sets, double batch_single_sets,
                       bool tuned);
// Clears the latch that a grid-barrier timeout sets on the current device's
// engines (they then use per-level launches); returns how many were cleared.
int engine_reset_persistent();

void engine_get_tuning(double &single_narrow_level_sets, double &single_wide_level_sets, double &batch_single_sets,
                       bool &tuned);

}  // namespace gqb
