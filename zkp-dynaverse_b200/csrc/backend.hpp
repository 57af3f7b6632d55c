// Owner ("backend") object behind the opaque void* of the C-ABI.
//
// Mirrors the reference owner (native/src/icicle_msm.cu:92-144), which is
// created on visible device 0; here it is created on the calling thread's
// current device (device 0 unless the caller chose another, e.g. one GPU per
// rank).  Used by one caller thread at a time, retired by any CUDA
// failure (later calls return -4), destroyed by dvgpu_backend_destroy.
// Unlike the reference it uses the device's primary context, so device
// pointers from other runtime users (e.g. torch) are valid in the
// device-pointer entry points; each owner has its own non-blocking stream and
// grow-only workspaces.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>

#include "../../include/dynaverse_gpu.h"
#include "batch.hpp"
#include "engine.hpp"
#include "g2.cuh"
#include "msm.cuh"
#include "ntt.cuh"

namespace dv {

struct ResidentBases {
    DevBuf points;  // Montgomery affine
    uint64_t n = 0;
    int g2 = 0;
    DevBuf pre_table;  // optional precomputed window multiples (n * pre_windows entries)
    int pre_c = 0, pre_windows = 0;
};

struct ResidentState;  // resident.cu
struct PolyState;      // poly.cu
struct PairingState;   // pairing.cu

struct Backend {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // device-to-host copies overlapping the main stream (lazy)
    bool retired = false;
    uint32_t large_bucket_factor = 0;
    std::string identity;

    MsmWorkspace msm;
    MsmStats msm_stats;
    NttWorkspace ntt;
    FixedBaseTables fixed_base;
    DevBuf in_points, in_scalars, conv_points, idx, out_buf, aux, err;
    PinnedBuf pin_in, pin_out, pin_err;
    DvgpuBatchStats batch_stats{};
    DvgpuSetupStats setup_stats{};
    DvgpuG2ValidationStats g2_stats{};
    DvgpuG2ValidationTraffic g2_traffic{};
    DvgpuG2KernelConfig g2_kernel{128, 0, 0, 0};
    DvgpuG2ExperimentStats g2_experiment{};
    int setup_mode = 2;
    int force_c = 0;
    int tuned_c_g1[40] = {};  // autotuned window width per ceil(log2(points per set))
    int tuned_c_g2[40] = {};

    std::map<uint64_t, std::unique_ptr<ResidentBases>> bases;
    std::map<uint64_t, std::unique_ptr<BatchPlan>> plans;  // CUDA-graph batch plans
    std::shared_ptr<ResidentState> resident;                // resident transactional buffers
    std::shared_ptr<PolyState> poly;                        // subproduct trees and polynomial scratch
    std::shared_ptr<PairingState> pairing;                  // prepared G2 points and pairing scratch
    uint64_t next_handle = 1;

    void release_all() noexcept;
    ~Backend() { release_all(); }
};

}  // namespace dv
