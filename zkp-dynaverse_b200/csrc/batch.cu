// Batch plans and the batched-NTT entry points (see batch.hpp).
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "abi_util.hpp"
#include "backend.hpp"
#include "batch.hpp"
#include "g2.cuh"

namespace dv {

void random_fr_launch(uint64_t seed, uint64_t n, uint8_t* d_out, cudaStream_t st);

namespace {

int ceil_log2(uint64_t n) {
    int k = 0;
    while ((1ull << k) < n) ++k;
    return k;
}

// Cost model of one class with precomputed tables, in mixed-addition
// units: every digit is one mixed addition; the reduction costs two full
// additions (2 x 1.4 mixed) per bucket and runs at about half the
// accumulation's efficiency.
int class_model_c(const BatchClass& k) {
    int best_c = 8;
    double best = 1e300;
    for (int c = 6; c <= 20; ++c) {
        const double W = (255 + c - 1) / c;
        const double cost = W * (double)k.total_n + 2.0 * 2.8 * (double)k.sets.size() * (double)(1u << (c - 1));
        if (cost < best) { best = cost; best_c = c; }
    }
    return best_c;
}

MsmPlan pre_plan(int c) { return MsmPlan{c, (255 + c - 1) / c, 1u << (c - 1), std::min(3, c - 1)}; }

void enqueue_class(BatchPlan& p, BatchClass& k, cudaStream_t st) {
    const MsmPrecomp<Fq> pre{k.table.view<G1A>(), k.plan.c, k.plan.windows};
    const SetMap map{k.set_off.view<uint32_t>(), k.set_src.view<uint32_t>(), (uint32_t)k.sets.size(), 1};
    msm_enqueue<Fq>(p.ws, nullptr, p.scalars.view<uint32_t>(), map, (uint32_t)k.total_n, k.plan, &pre,
                    p.err.view<uint32_t>(), st);
    msm_finish_device<Fq>(p.ws.windows.view<XYZZ<Fq>>(), (uint32_t)k.sets.size(), 1, k.plan.c,
                          k.out_idx.view<uint32_t>(), p.msm_out.view<uint8_t>(), st);
}

// Enqueues the whole plan on p.stream (NTTs forked onto p.side).
void enqueue_msms(BatchPlan& p) {
    DV_CUDA(cudaMemsetAsync(p.err.view<uint32_t>(), 0xff, sizeof(uint32_t), p.stream));
    for (auto& k : p.classes) enqueue_class(p, *k, p.stream);
}

void enqueue_all(BatchPlan& p) {
    const bool ntts = p.ntt.count > 0;
    if (ntts) {
        DV_CUDA(cudaEventRecord(p.fork, p.stream));
        DV_CUDA(cudaStreamWaitEvent(p.side, p.fork, 0));
        ntt_batch_enqueue(p.ntt, p.side);
        DV_CUDA(cudaEventRecord(p.join, p.side));
    }
    enqueue_msms(p);
    if (ntts) DV_CUDA(cudaStreamWaitEvent(p.stream, p.join, 0));
}

double time_class(BatchPlan& p, BatchClass& k, int reps) {
    cudaEvent_t e0, e1;
    DV_CUDA(cudaEventCreate(&e0));
    DV_CUDA(cudaEventCreate(&e1));
    enqueue_class(p, k, p.stream);  // warm-up (sizes the workspace)
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        DV_CUDA(cudaEventRecord(e0, p.stream));
        enqueue_class(p, k, p.stream);
        DV_CUDA(cudaEventRecord(e1, p.stream));
        DV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        DV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// Best of `reps` timed runs of the plan's NTT batch alone on p.stream.
double time_ntt(BatchPlan& p, int reps) {
    cudaEvent_t e0, e1;
    DV_CUDA(cudaEventCreate(&e0));
    DV_CUDA(cudaEventCreate(&e1));
    ntt_batch_enqueue(p.ntt, p.stream);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        DV_CUDA(cudaEventRecord(e0, p.stream));
        ntt_batch_enqueue(p.ntt, p.stream);
        DV_CUDA(cudaEventRecord(e1, p.stream));
        DV_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        DV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// Weight of word i in the output hash: the splitmix64 finaliser of i
// (Steele, Lea, Flood 2014), odd so that no word's low bits are lost.
DV_INL uint64_t word_weight(uint64_t i) {
    uint64_t z = i + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (z ^ (z >> 31)) | 1ull;
}

// out += sum over the n 32-bit words w_i of w_i * word_weight(i) (mod 2^64):
// independent of the order of the additions, so two arrays with the same
// words give the same value and a difference anywhere changes it except
// with negligible probability.
__global__ void k_words_hash(const uint4* __restrict__ a, uint64_t n16, unsigned long long* out) {
    uint64_t h = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint4 x = a[i];
        h += x.x * word_weight(4 * i) + x.y * word_weight(4 * i + 1) + x.z * word_weight(4 * i + 2) +
             x.w * word_weight(4 * i + 3);
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) h += __shfl_down_sync(0xffffffffu, h, d);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)h);
}

// Picks the batch NTT's tile (2^10, 2^11 or 2^12 elements: 32, 64 or 128 KB
// of shared memory, hence fewer or more passes and resident blocks) and
// register round (radix 2, 4 or 8) by timing each pair on the plan's own
// transforms.  Every candidate's outputs must hash to the first
// candidate's (a 64-bit position-weighted sum of the output words, so no
// second copy of the outputs is held); a disagreement fails the plan.
// Returns the candidates as JSON.
std::string tune_ntt(BatchPlan& p, const std::vector<NttBatchItem>& items, const uint8_t* d_out) {
    const uint64_t n16 = 2 * p.ntt_elements;  // 16-byte words of the outputs
    DevBuf hash;
    unsigned long long* d_hash = hash.as<unsigned long long>(1);
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n16 + 255) / 256, 4ull * sm_count()));
    unsigned long long first = 0;
    bool have_first = false;
    std::string cands;
    double best_ms = 1e300;
    int best_t = BATCH_TILE_DEFAULT, best_r = 0;
    for (int t = 10; t <= BATCH_TILE_MAX; ++t) {
        ntt_batch_prepare(p.ntt_ws, p.ntt, items, p.stream, t);
        for (int r = 1; r <= 3; ++r) {
            ntt_batch_set_radix(p.ntt, r);
            const double ms = time_ntt(p, 3);
            ntt_batch_check(p.ntt, p.stream);
            unsigned long long h = 0;
            DV_CUDA(cudaMemsetAsync(d_hash, 0, sizeof(unsigned long long), p.stream));
            k_words_hash<<<grid, 256, 0, p.stream>>>((const uint4*)d_out, n16, d_hash);
            DV_LAUNCH();
            DV_CUDA(cudaMemcpyAsync(&h, d_hash, sizeof(h), cudaMemcpyDeviceToHost, p.stream));
            DV_CUDA(cudaStreamSynchronize(p.stream));
            if (!have_first) {
                first = h;
                have_first = true;
            } else if (h != first) {
                throw CudaFailure("batch NTT tile 2^" + std::to_string(t) + " radix " + std::to_string(1 << r) +
                                  " disagrees with the first candidate");
            }
            cands += std::string(cands.empty() ? "" : ",") + "{\"tile\":" + std::to_string(1 << t) +
                     ",\"radix\":" + std::to_string(1 << r) + ",\"grid\":" + std::to_string(p.ntt.grid) +
                     ",\"tiles\":" + std::to_string(p.ntt.ntiles) + ",\"ms\":" + std::to_string(ms) + "}";
            if (ms < best_ms) {
                best_ms = ms;
                best_t = t;
                best_r = r;
            }
        }
    }
    ntt_batch_prepare(p.ntt_ws, p.ntt, items, p.stream, best_t);
    ntt_batch_set_radix(p.ntt, best_r);
    return cands;
}

}  // namespace

BatchPlan::~BatchPlan() {
    if (stream) cudaStreamSynchronize(stream);
    if (side) cudaStreamSynchronize(side);
    if (copy) cudaStreamSynchronize(copy);
    if (last && last != stream && last != side) cudaStreamSynchronize(last);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (exec_msm) cudaGraphExecDestroy(exec_msm);
    if (graph_msm) cudaGraphDestroy(graph_msm);
    if (exec_ntt) cudaGraphExecDestroy(exec_ntt);
    if (graph_ntt) cudaGraphDestroy(graph_ntt);
    if (ntt_ready) cudaEventDestroy(ntt_ready);
    if (ntt_done) cudaEventDestroy(ntt_done);
    if (copy) cudaStreamDestroy(copy);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
}

std::unique_ptr<BatchPlan> batch_plan_create(const Affine<Fq>* points, uint64_t n_points,
                                             const std::vector<uint64_t>& msm_sizes,
                                             const std::vector<uint32_t>& ntt_logs,
                                             const std::vector<int32_t>& ntt_kinds, std::string& log) {
    auto plan = std::make_unique<BatchPlan>();
    BatchPlan& p = *plan;
    DV_CUDA(cudaGetDevice(&p.device));
    DV_CUDA(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
    DV_CUDA(cudaStreamCreateWithFlags(&p.side, cudaStreamNonBlocking));
    DV_CUDA(cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming));
    DV_CUDA(cudaEventCreateWithFlags(&p.join, cudaEventDisableTiming));
    DV_CUDA(cudaStreamCreateWithFlags(&p.copy, cudaStreamNonBlocking));
    DV_CUDA(cudaEventCreateWithFlags(&p.ntt_ready, cudaEventDisableTiming));
    DV_CUDA(cudaEventCreateWithFlags(&p.ntt_done, cudaEventDisableTiming));

    // ---- MSM sets: offsets in the scalar array, size classes
    p.msm_sizes = msm_sizes;
    p.scalar_off.resize(msm_sizes.size());
    std::map<int, std::vector<uint32_t>> by_band;
    for (size_t i = 0; i < msm_sizes.size(); ++i) {
        const uint64_t n = msm_sizes[i];
        if (n < 1 || n > n_points) throw InvalidArgument("batch MSM size out of range of the registered bases");
        p.scalar_off[i] = p.total_scalars;
        p.total_scalars += n;
        by_band[(ceil_log2(n) + 1) / 2].push_back((uint32_t)i);
    }
    if (p.total_scalars > 0xffffffffull / 32) throw InvalidArgument("batch has too many scalars");
    p.scalars.as<uint8_t>(std::max<uint64_t>(1, p.total_scalars) * 32);
    p.msm_out.as<uint8_t>(std::max<size_t>(1, msm_sizes.size()) * 64);
    p.err.as<uint32_t>(1);
    if (p.total_scalars) random_fr_launch(0xba7c4ull, p.total_scalars, p.scalars.view<uint8_t>(), p.stream);

    // ---- NTTs
    p.ntt_logs = ntt_logs;
    p.ntt_kinds = ntt_kinds;
    for (uint32_t L : ntt_logs) {
        if (L < 1 || L > 24) throw InvalidArgument("batch NTT size must be 2^1..2^24");
        p.ntt_off.push_back(p.ntt_elements);
        p.ntt_elements += 1ull << L;
    }
    uint8_t* nin = p.ntt_in.as<uint8_t>(std::max<uint64_t>(1, p.ntt_elements) * 32);
    uint8_t* nout = p.ntt_out.as<uint8_t>(std::max<uint64_t>(1, p.ntt_elements) * 32);
    if (p.ntt_elements) random_fr_launch(0x7711ull, p.ntt_elements, nin, p.stream);
    std::vector<NttBatchItem> items;
    for (size_t j = 0; j < ntt_logs.size(); ++j)
        items.push_back(NttBatchItem{nin + 32 * p.ntt_off[j], nout + 32 * p.ntt_off[j], (int)ntt_logs[j],
                                     ntt_kinds.empty() ? 0 : (int)ntt_kinds[j]});
    ntt_batch_prepare(p.ntt_ws, p.ntt, items, p.stream);
    const std::string ntt_cands = p.ntt.count ? tune_ntt(p, items, nout) : std::string();

    // ---- classes: set maps, autotuned window width, precomputed table
    log = "{\"classes\":[";
    bool first_class = true;
    for (auto& band : by_band) {
        auto k = std::make_unique<BatchClass>();
        k->sets = band.second;
        std::vector<uint32_t> off(1, 0), src, out;
        for (uint32_t i : k->sets) {
            const uint64_t n = msm_sizes[i];
            k->max_n = std::max<uint32_t>(k->max_n, (uint32_t)n);
            k->total_n += n;
            off.push_back((uint32_t)k->total_n);
            src.push_back((uint32_t)p.scalar_off[i]);
            out.push_back(i);
        }
        const uint32_t cnt = (uint32_t)k->sets.size();
        DV_CUDA(cudaMemcpyAsync(k->set_off.as<uint32_t>(cnt + 1), off.data(), (cnt + 1) * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, p.stream));
        DV_CUDA(cudaMemcpyAsync(k->set_src.as<uint32_t>(cnt), src.data(), cnt * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, p.stream));
        DV_CUDA(cudaMemcpyAsync(k->out_idx.as<uint32_t>(cnt), out.data(), cnt * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, p.stream));
        DV_CUDA(cudaStreamSynchronize(p.stream));  // the host vectors die with this iteration

        const int model = class_model_c(*k);
        std::string cands;
        double best_ms = 1e300;
        int best_c = 0;
        DevBuf spare;  // table of the candidate that is not (yet) the best
        for (int c = std::max(6, model - 1); c <= std::min(20, model + 1); ++c) {
            const MsmPlan pl = pre_plan(c);
            if ((uint64_t)cnt * pl.buckets > (1ull << 26) || k->total_n * (uint64_t)pl.windows >= (1ull << 31))
                continue;
            // build the candidate's table in the spare buffer and try it
            msm_precompute<Fq>(points, k->max_n, c, pl.windows, spare.as<G1A>((uint64_t)k->max_n * pl.windows),
                               p.stream);
            std::swap(spare.ptr, k->table.ptr);
            std::swap(spare.cap, k->table.cap);
            k->plan = pl;
            const double ms = time_class(p, *k, 2);
            cands += std::string(cands.empty() ? "" : ",") + "{\"c\":" + std::to_string(c) +
                     ",\"ms\":" + std::to_string(ms) + "}";
            if (ms < best_ms) {
                best_ms = ms;
                best_c = c;
            } else {
                // the earlier best stays: swap its table back
                std::swap(spare.ptr, k->table.ptr);
                std::swap(spare.cap, k->table.cap);
                k->plan = pre_plan(best_c);
            }
        }
        if (!best_c) throw InvalidArgument("batch MSM class too large for one launch sequence");
        spare.release();
        k->plan = pre_plan(best_c);
        // bucket partition of the reduction: segments of 2^s buckets around
        // the rule's choice (the class's c above was timed with the rule's)
        const int rule = msm_seg_log((uint64_t)cnt * k->plan.buckets, k->plan.buckets, best_c, true);
        std::string seg_cands = "{\"seg\":" + std::to_string(1 << rule) + ",\"ms\":" + std::to_string(best_ms) + "}";
        int best_seg = 0;
        for (int sg = std::max(1, rule - 1); sg <= std::min(best_c - 1, rule + 1); ++sg) {
            if (sg == rule) continue;
            k->plan.seg_force = sg;
            const double ms = time_class(p, *k, 2);
            seg_cands += ",{\"seg\":" + std::to_string(1 << sg) + ",\"ms\":" + std::to_string(ms) + "}";
            if (ms < best_ms) {
                best_ms = ms;
                best_seg = sg;
            }
        }
        k->plan.seg_force = best_seg;  // 0: the rule's
        log += std::string(first_class ? "" : ",") + "{\"sets\":" + std::to_string(cnt) +
               ",\"max_points\":" + std::to_string(k->max_n) + ",\"points\":" + std::to_string(k->total_n) +
               ",\"model_c\":" + std::to_string(model) + ",\"candidates\":[" + cands +
               "],\"best_c\":" + std::to_string(best_c) + ",\"seg_candidates\":[" + seg_cands +
               "],\"best_seg\":" + std::to_string(1 << (best_seg ? best_seg : rule)) +
               ",\"best_ms\":" + std::to_string(best_ms) +
               ",\"table_bytes\":" + std::to_string((uint64_t)k->max_n * k->plan.windows * sizeof(G1A)) + "}";
        first_class = false;
        p.classes.push_back(std::move(k));
    }
    log += "],\"ntt\":{\"transforms\":" + std::to_string(p.ntt.count) +
           ",\"elements\":" + std::to_string(p.ntt.elements) + ",\"tiles\":" + std::to_string(p.ntt.ntiles) +
           ",\"grid\":" + std::to_string(p.ntt.grid) + ",\"candidates\":[" + ntt_cands +
           "],\"best_tile\":" + std::to_string(1 << p.ntt.tile_log) +
           ",\"best_radix\":" + std::to_string(1 << p.ntt.radix_log) + "}";

    // ---- one uncaptured run (final workspace sizes), then capture
    enqueue_all(p);
    DV_CUDA(cudaStreamSynchronize(p.stream));
    DV_CUDA(cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue_all(p);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(p.stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    DV_CUDA(cudaStreamEndCapture(p.stream, &p.graph));
    DV_CUDA(cudaGraphInstantiate(&p.exec, p.graph, 0));
    DV_CUDA(cudaGraphGetNodes(p.graph, nullptr, &p.graph_nodes));
    std::vector<cudaGraphNode_t> nodes(p.graph_nodes);
    DV_CUDA(cudaGraphGetNodes(p.graph, nodes.data(), &p.graph_nodes));
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        DV_CUDA(cudaGraphNodeGetType(node, &type));
        if (type == cudaGraphNodeTypeKernel) ++p.graph_kernels;
    }
    // the two halves alone, for host-buffer runs
    if (!p.classes.empty()) {
        DV_CUDA(cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_msms(p);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(p.stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        DV_CUDA(cudaStreamEndCapture(p.stream, &p.graph_msm));
        DV_CUDA(cudaGraphInstantiate(&p.exec_msm, p.graph_msm, 0));
    }
    if (p.ntt.count) {
        DV_CUDA(cudaStreamBeginCapture(p.side, cudaStreamCaptureModeThreadLocal));
        try {
            ntt_batch_enqueue(p.ntt, p.side);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(p.side, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        DV_CUDA(cudaStreamEndCapture(p.side, &p.graph_ntt));
        DV_CUDA(cudaGraphInstantiate(&p.exec_ntt, p.graph_ntt, 0));
    }
    log += ",\"graph_nodes\":" + std::to_string(p.graph_nodes) +
           ",\"graph_kernels\":" + std::to_string(p.graph_kernels) + "}";
    p.last = p.stream;
    return plan;
}

void batch_plan_launch(BatchPlan& p, cudaStream_t st) {
    p.last = st ? st : p.stream;
    DV_CUDA(cudaGraphLaunch(p.exec, p.last));
}

void batch_plan_run_host(BatchPlan& p, const uint8_t* scalars, const uint8_t* ntt_values, uint8_t* msm_results,
                         uint8_t* ntt_results) {
    const bool msms = p.total_scalars > 0, ntts = p.ntt_elements > 0;
    if (msms) {
        DV_CUDA(cudaMemcpyAsync(p.scalars.view<uint8_t>(), scalars, p.total_scalars * 32, cudaMemcpyHostToDevice,
                                p.stream));
        DV_CUDA(cudaMemsetAsync(p.err.view<uint32_t>(), 0xff, sizeof(uint32_t), p.stream));
        fixed_base_validate(p.scalars.view<uint8_t>(), p.total_scalars, p.err.view<uint32_t>(), p.stream);
        uint32_t bad = 0;
        DV_CUDA(cudaMemcpyAsync(&bad, p.err.view<uint32_t>(), sizeof(uint32_t), cudaMemcpyDeviceToHost, p.stream));
        DV_CUDA(cudaStreamSynchronize(p.stream));
        if (bad != 0xffffffffu) throw InvalidArgument("non-canonical scalar at index " + std::to_string(bad));
        DV_CUDA(cudaGraphLaunch(p.exec_msm, p.stream));
    }
    if (ntts) {
        DV_CUDA(cudaMemcpyAsync(p.ntt_in.view<uint8_t>(), ntt_values, p.ntt_elements * 32, cudaMemcpyHostToDevice,
                                p.copy));
        DV_CUDA(cudaEventRecord(p.ntt_ready, p.copy));
        DV_CUDA(cudaStreamWaitEvent(p.side, p.ntt_ready, 0));
        DV_CUDA(cudaGraphLaunch(p.exec_ntt, p.side));
        DV_CUDA(cudaEventRecord(p.ntt_done, p.side));
        try {
            ntt_batch_check(p.ntt, p.side);  // waits for the NTTs only
        } catch (...) {
            cudaStreamSynchronize(p.stream);  // leave the plan idle
            throw;
        }
        DV_CUDA(cudaMemcpyAsync(ntt_results, p.ntt_out.view<uint8_t>(), p.ntt_elements * 32, cudaMemcpyDeviceToHost,
                                p.copy));
    }
    if (msms) {
        DV_CUDA(cudaStreamSynchronize(p.stream));
        uint32_t bad = 0;
        DV_CUDA(cudaMemcpy(&bad, p.err.view<uint32_t>(), sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (bad != 0xffffffffu) throw InvalidArgument("non-canonical scalar at index " + std::to_string(bad));
        DV_CUDA(cudaMemcpyAsync(msm_results, p.msm_out.view<uint8_t>(), p.msm_sizes.size() * 64,
                                cudaMemcpyDeviceToHost, p.copy));
    }
    DV_CUDA(cudaStreamSynchronize(p.copy));
    p.last = p.stream;
}

void batch_plan_check(BatchPlan& p) {
    DV_CUDA(cudaStreamSynchronize(p.last));
    uint32_t bad = 0;
    DV_CUDA(cudaMemcpy(&bad, p.err.view<uint32_t>(), sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (bad != 0xffffffffu) throw InvalidArgument("non-canonical scalar at index " + std::to_string(bad));
    ntt_batch_check(p.ntt, p.last);
}

}  // namespace dv

using namespace dv;

namespace {

std::vector<NttBatchItem> batch_items(const uint8_t* in, uint8_t* out, const uint32_t* logs, const int32_t* kinds,
                                      size_t count) {
    std::vector<NttBatchItem> items;
    uint64_t total = 0;
    for (size_t i = 0; i < count; ++i) {
        require(logs[i] >= 1 && logs[i] <= 24, "batch NTT size must be 2^1..2^24");
        const int kind = kinds ? kinds[i] : 0;
        require(kind >= 0 && kind <= 3, "invalid NTT kind");
        items.push_back(NttBatchItem{in + 32 * total, out + 32 * total, (int)logs[i], kind});
        total += 1ull << logs[i];
    }
    return items;
}

BatchPlan& plan_of(Backend& b, uint64_t handle) {
    auto it = b.plans.find(handle);
    require(it != b.plans.end(), "unknown batch plan handle");
    return *it->second;
}

}  // namespace

extern "C" int dvgpu_bn254_ntt_batch_device(void* opaque, const uint8_t* d_values, const uint32_t* log_sizes,
                                            const int32_t* kinds, size_t count, uint8_t* d_results, void* stream,
                                            char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(!count || (log_sizes && d_values && d_results), "invalid batch NTT arguments");
        const auto items = batch_items(d_values, d_results, log_sizes, kinds, count);
        if (!count) return;
        const cudaStream_t st = pick(b, stream);
        NttBatch batch;
        ntt_batch_prepare(b.ntt, batch, items, st);
        ntt_batch_enqueue(batch, st);
        ntt_batch_check(batch, st);
    });
}

extern "C" int dvgpu_bn254_ntt_batch(void* opaque, const uint8_t* values, const uint32_t* log_sizes,
                                     const int32_t* kinds, size_t count, uint8_t* results, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(!count || (log_sizes && values && results), "invalid batch NTT arguments");
        uint64_t total = 0;
        for (size_t i = 0; i < count; ++i) {
            require(log_sizes[i] >= 1 && log_sizes[i] <= 24, "batch NTT size must be 2^1..2^24");
            total += 1ull << log_sizes[i];
        }
        if (!count) return;
        uint8_t* d = b.in_scalars.as<uint8_t>(total * 32);
        const auto items = batch_items(d, d, log_sizes, kinds, count);
        DV_CUDA(cudaMemcpyAsync(d, values, total * 32, cudaMemcpyHostToDevice, b.stream));
        NttBatch batch;
        ntt_batch_prepare(b.ntt, batch, items, b.stream);
        ntt_batch_enqueue(batch, b.stream);
        ntt_batch_check(batch, b.stream);
        DV_CUDA(cudaMemcpyAsync(results, d, total * 32, cudaMemcpyDeviceToHost, b.stream));
        DV_CUDA(cudaStreamSynchronize(b.stream));
    });
}

extern "C" int dvgpu_batch_plan_create(void* opaque, uint64_t bases_handle, const uint64_t* msm_sizes,
                                       size_t msm_count, const uint32_t* ntt_log_sizes, const int32_t* ntt_kinds,
                                       size_t ntt_count, uint64_t* plan, char* log_json, size_t log_capacity,
                                       char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(plan && (!msm_count || msm_sizes) && (!ntt_count || ntt_log_sizes) && (msm_count || ntt_count),
                "invalid batch plan arguments");
        require(msm_count <= DVGPU_MAX_MSM_BATCH_SIZE && ntt_count <= DVGPU_MAX_MSM_BATCH_SIZE,
                "too many batch items");
        const Affine<Fq>* pts = nullptr;
        uint64_t npts = 0;
        if (msm_count) {
            auto it = b.bases.find(bases_handle);
            require(it != b.bases.end(), "unknown base handle");
            require(!it->second->g2, "batch plans take G1 bases");
            pts = it->second->points.view<G1A>();
            npts = it->second->n;
        }
        if (ntt_kinds)
            for (size_t j = 0; j < ntt_count; ++j) require(ntt_kinds[j] >= 0 && ntt_kinds[j] <= 3, "invalid NTT kind");
        std::string log;
        auto p = batch_plan_create(pts, npts, std::vector<uint64_t>(msm_sizes, msm_sizes + msm_count),
                                   std::vector<uint32_t>(ntt_log_sizes, ntt_log_sizes + ntt_count),
                                   ntt_kinds ? std::vector<int32_t>(ntt_kinds, ntt_kinds + ntt_count)
                                             : std::vector<int32_t>(),
                                   log);
        const uint64_t h = b.next_handle++;
        b.plans[h] = std::move(p);
        *plan = h;
        if (log_json && log_capacity) {
            const size_t k = std::min(log_capacity - 1, log.size());
            memcpy(log_json, log.data(), k);
            log_json[k] = '\0';
        }
    });
}

extern "C" int dvgpu_batch_plan_buffers(void* opaque, uint64_t handle, DvgpuBatchPlanBuffers* out, char* error,
                                        size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(out, "null output");
        BatchPlan& p = plan_of(b, handle);
        out->scalars = p.scalars.view<uint8_t>();
        out->ntt_values = p.ntt_in.view<uint8_t>();
        out->msm_results = p.msm_out.view<uint8_t>();
        out->ntt_results = p.ntt_out.view<uint8_t>();
        out->scalar_bytes = p.total_scalars * 32;
        out->ntt_bytes = p.ntt_elements * 32;
        out->msm_result_bytes = p.msm_sizes.size() * 64;
        out->msm_classes = (uint32_t)p.classes.size();
        out->graph_nodes = (uint32_t)p.graph_nodes;
        out->graph_kernels = (uint32_t)p.graph_kernels;
        out->reserved = 0;
    });
}

extern "C" int dvgpu_batch_plan_launch(void* opaque, uint64_t handle, void* stream, char* error, size_t cap) {
    return guarded(opaque, error, cap,
                   [&](Backend& b) { batch_plan_launch(plan_of(b, handle), static_cast<cudaStream_t>(stream)); });
}

extern "C" int dvgpu_batch_plan_check(void* opaque, uint64_t handle, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) { batch_plan_check(plan_of(b, handle)); });
}

extern "C" int dvgpu_batch_plan_run(void* opaque, uint64_t handle, const uint8_t* scalars, const uint8_t* ntt_values,
                                    uint8_t* msm_results, uint8_t* ntt_results, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        BatchPlan& p = plan_of(b, handle);
        require((!p.total_scalars || (scalars && msm_results)) && (!p.ntt_elements || (ntt_values && ntt_results)),
                "invalid batch plan buffers");
        batch_plan_run_host(p, scalars, ntt_values, msm_results, ntt_results);
    });
}

extern "C" int dvgpu_batch_plan_destroy(void* opaque, uint64_t handle, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        plan_of(b, handle);
        b.plans.erase(handle);
    });
}
