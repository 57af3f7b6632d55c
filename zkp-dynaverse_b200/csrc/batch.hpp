// Batch plans: a fixed workload of G1 MSMs over prefixes of one resident
// base set plus NTTs of fixed sizes, captured once into a CUDA graph.
//
// The reference batches MSMs by padding every set to the next power of two
// and grouping 64 sets per ICICLE call (crates/gpu/src/icicle.rs:281-339,
// native/src/icicle_msm.cu:810-880), and runs one NTT call per vector
// (icicle.rs:429-456).  A plan instead
//   - groups the MSMs into size classes (bands of two in ceil(log2 n)); each
//     class is one launch sequence over all its sets with its own window
//     width c, picked by timing candidates (the autotuner), and its own
//     table of precomputed window multiples over the prefix the class needs,
//     so every set has one bucket set and no window combination;
//   - finishes the MSMs on the device (affine normalisation, results in
//     request order), so nothing returns to the host mid-graph;
//   - runs every NTT in one persistent launch on a parallel branch;
//   - captures all of it once and replays the graph per run.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"
#include "msm.cuh"
#include "ntt.cuh"

namespace dv {

struct BatchClass {
    std::vector<uint32_t> sets;  // request indices, in launch order
    uint32_t max_n = 0;          // longest prefix of the class
    uint64_t total_n = 0;        // scalars of the class
    MsmPlan plan{};
    DevBuf table;                // max_n * windows precomputed window multiples
    DevBuf set_off, set_src, out_idx;
};

struct BatchPlan {
    int device = 0;
    cudaStream_t stream = nullptr, side = nullptr, last = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // host-buffer runs: the MSM and NTT halves as separate graphs, a copy
    // stream and the events that order them
    cudaStream_t copy = nullptr;
    cudaEvent_t ntt_ready = nullptr, ntt_done = nullptr;
    cudaGraph_t graph_msm = nullptr, graph_ntt = nullptr;
    cudaGraphExec_t exec_msm = nullptr, exec_ntt = nullptr;
    size_t graph_nodes = 0, graph_kernels = 0;

    std::vector<uint64_t> msm_sizes, scalar_off;
    std::vector<std::unique_ptr<BatchClass>> classes;
    uint64_t total_scalars = 0;
    MsmWorkspace ws;

    std::vector<uint32_t> ntt_logs;
    std::vector<int32_t> ntt_kinds;
    std::vector<uint64_t> ntt_off;
    uint64_t ntt_elements = 0;
    NttWorkspace ntt_ws;
    NttBatch ntt;

    DevBuf scalars, ntt_in, ntt_out, msm_out, err;

    ~BatchPlan();
};

// Builds the plan (autotuning each class, building its table), runs it once
// uncaptured, then captures and instantiates the graph.  points: the
// registered bases in Montgomery affine form (n_points of them); every MSM
// size must be within 1..n_points.  log receives the autotuner's JSON.
std::unique_ptr<BatchPlan> batch_plan_create(const Affine<Fq>* points, uint64_t n_points,
                                             const std::vector<uint64_t>& msm_sizes,
                                             const std::vector<uint32_t>& ntt_logs,
                                             const std::vector<int32_t>& ntt_kinds, std::string& log);
// Enqueues one replay on `stream` (the plan's own stream when null).
void batch_plan_launch(BatchPlan& plan, cudaStream_t stream);
// Waits for the last replay; throws InvalidArgument for invalid inputs.
void batch_plan_check(BatchPlan& plan);
// One run from host buffers: scalars up and checked first (no output is
// written on a bad input), the MSM graph on them while the NTT inputs go up,
// the NTT graph beside the MSMs, its outputs down while the MSMs run.
void batch_plan_run_host(BatchPlan& plan, const uint8_t* scalars, const uint8_t* ntt_values, uint8_t* msm_results,
                         uint8_t* ntt_results);

}  // namespace dv
