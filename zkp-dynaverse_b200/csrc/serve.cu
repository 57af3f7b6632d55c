// Serving engine: commitment updates from many sessions, continuously batched.
//
// The reference serves Dynaverse updates one call at a time per session
// (crates/protocol/src/session.rs:51-142; every update re-enters the
// operator backend, crates/protocol/src/sparse.rs:79-276, whose sparse MSMs
// go through msm_sparse_batch one request at a time).  Its operator-level
// core is the commitment update of a sparse edit: for a session with SRS
// bases G_i and committed vector v, rewriting the entries of a support I
// with new values v'_i changes the commitment by
//      C' = C + sum_{i in I} (v'_i - v_i) G_i ,
// a sparse MSM over the session's bases.  This engine keeps each session's
// bases, vector and commitment resident, admits sessions against a stated
// HBM budget, and on one engine thread merges the pending requests of many
// sessions into shared launches: one gather-and-delta kernel and one
// multi-set MSM launch sequence per batch.  Requests that arrive while a
// batch is on the GPU form the next batch (continuous batching).  The same
// engine with batches of one request is the per-call form.
//
// Each session also keeps a table of precomputed window multiples of its
// bases (c = 8, 32 windows: 2 KB per base), so a request's MSM adds every
// window into one set of 128 buckets and needs no window combination; the
// batch's sets are finished (normalised) on the device.
//
// Within a batch a session has at most one request (later requests of a
// session wait for the next batch), so each request's deltas are taken
// against the vector its predecessors left and every result equals the one
// the request gets alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <future>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/dynaverse_gpu.h"
#include "curve.cuh"
#include "host_curve.hpp"
#include "msm.cuh"

namespace dv {
namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Canonical Fr check on little-endian bytes (value < r).
bool fr_canonical(const uint8_t* b) {
    static const uint64_t R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                                  0x30644e72e131a029ull};
    uint64_t w[4];
    memcpy(w, b, 32);
    for (int i = 3; i >= 0; --i) {
        if (w[i] < R[i]) return true;
        if (w[i] > R[i]) return false;
    }
    return false;
}

// Canonical affine G1 bytes (x || y, all-zero = infinity) -> host XYZZ.
dvh::XYZZ<dvh::Fq> xyzz_of(const uint8_t* p) {
    bool zero = true;
    for (int i = 0; i < 64; ++i) zero &= p[i] == 0;
    if (zero) return dvh::xyzz_inf<dvh::Fq>();
    uint64_t x[4], y[4];
    memcpy(x, p, 32);
    memcpy(y, p + 32, 32);
    return {dvh::from_canonical(x), dvh::from_canonical(y), dvh::one(), dvh::one()};
}

constexpr int SERVE_C = 8;
constexpr int SERVE_W = (255 + SERVE_C - 1) / SERVE_C;  // 32 windows

// Request of update entry e: the largest r with req_off[r] <= e.
DV_INL uint32_t serve_request_of(uint32_t e, const uint32_t* __restrict__ req_off, uint32_t count) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (req_off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

// One thread per (update entry, window): find the entry's request, gather
// the window multiple 2^(c w) G_i from the session's table; the window-0
// thread also emits the delta new - old (mod r) as the MSM scalar.  The
// resident values are not touched here: k_serve_commit writes them once the
// batch's MSM has completed.
__global__ void k_serve_prepare(uint32_t total, const uint32_t* __restrict__ req_off, uint32_t count,
                                const G1A* const* __restrict__ tables, uint8_t* const* __restrict__ values,
                                const uint32_t* __restrict__ idx, const uint8_t* __restrict__ new_vals,
                                G1A* __restrict__ gathered, uint8_t* __restrict__ deltas) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)total * SERVE_W) return;
    const uint32_t e = (uint32_t)(t / SERVE_W), w = (uint32_t)(t % SERVE_W);
    const uint32_t r = serve_request_of(e, req_off, count);
    const uint32_t i = idx[e];
    gathered[t] = tables[r][(uint64_t)i * SERVE_W + w];
    if (w) return;
    Fr oldv, newv;
    load_words(values[r] + 32ull * i, oldv.v);
    load_words(new_vals + 32ull * e, newv.v);
    const Fr d = Fr::sub(newv, oldv);  // canonical operands: canonical difference
    store_words(deltas + 32ull * e, d.v);
}

// After a successful batch: the resident values take the new ones.
__global__ void k_serve_commit(uint32_t total, const uint32_t* __restrict__ req_off, uint32_t count,
                               uint8_t* const* __restrict__ values, const uint32_t* __restrict__ idx,
                               const uint8_t* __restrict__ new_vals) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const uint32_t r = serve_request_of(e, req_off, count);
    uint32_t w[8];
    load_words(new_vals + 32ull * e, w);
    store_words(values[r] + 32ull * idx[e], w);
}

struct Session {
    uint64_t id = 0, n = 0, footprint = 0;
    DevBuf srs, table, values;
    uint8_t commitment[64] = {};
};

struct Request {
    uint64_t ticket = 0, session = 0, submit_ns = 0;
    std::vector<uint32_t> idx;
    std::vector<uint8_t> vals;
};

struct Outcome {
    bool ready = false;
    int status = 0;
    std::string error;
    uint8_t commitment[64] = {};
    DvgpuServeResult res{};
};

class Server {
public:
    Server(uint64_t budget, uint32_t max_batch) : budget_(budget), max_batch_(std::max<uint32_t>(1, max_batch)) {
        DV_CUDA(cudaGetDevice(&device_));
        worker_ = std::thread([this] { loop(); });
        run([this] { DV_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
    }

    uint64_t open_session(const uint8_t* srs_wire, const uint8_t* values, uint64_t n, uint8_t* commitment) {
        uint64_t id = 0;
        run([&] {
            const uint64_t footprint = n * (sizeof(G1A) * (1 + SERVE_W) + 32) + 64;
            if (resident_ + footprint > budget_)
                throw InvalidArgument("session does not fit the HBM budget (" + std::to_string(resident_) + " + " +
                                      std::to_string(footprint) + " > " + std::to_string(budget_) + " bytes)");
            auto s = std::make_unique<Session>();
            s->n = n;
            s->footprint = footprint;
            uint8_t* wire = stage_.as<uint8_t>(n * 64);
            DV_CUDA(cudaMemcpyAsync(wire, srs_wire, n * 64, cudaMemcpyHostToDevice, stream_));
            uint32_t* bad = err_.as<uint32_t>(1);
            DV_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), stream_));
            convert_points<Fq>(wire, s->srs.as<G1A>(n), n, bad, stream_);
            uint8_t* vals = s->values.as<uint8_t>(n * 32);
            DV_CUDA(cudaMemcpyAsync(vals, values, n * 32, cudaMemcpyHostToDevice, stream_));
            uint32_t h_bad = 0;
            DV_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
            DV_CUDA(cudaStreamSynchronize(stream_));
            if (h_bad != 0xffffffffu) throw InvalidArgument("invalid SRS point at index " + std::to_string(h_bad));
            msm_precompute<Fq>(s->srs.view<G1A>(), n, SERVE_C, SERVE_W, s->table.as<G1A>(n * SERVE_W), stream_);
            const uint32_t offs[2] = {0u, (uint32_t)n};
            msm_run<Fq>(ws_, s->srs.view<G1A>(), s->values.view<uint32_t>(), offs, 1, 0, stream_, s->commitment,
                        nullptr);
            memcpy(commitment, s->commitment, 64);
            std::lock_guard<std::mutex> lk(mu_);
            s->id = id = next_session_++;
            resident_ += footprint;
            sessions_[id] = std::move(s);
        });
        return id;
    }

    void close_session(uint64_t id) {
        run([&] {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = sessions_.find(id);
            if (it == sessions_.end()) throw InvalidArgument("unknown session");
            for (const Request& r : queue_)
                if (r.session == id) throw InvalidArgument("session has pending requests");
            resident_ -= it->second->footprint;
            sessions_.erase(it);
        });
    }

    uint64_t submit(uint64_t session, const uint64_t* idx, const uint8_t* vals, size_t k) {
        Request r;
        r.submit_ns = now_ns();
        r.session = session;
        r.idx.resize(k);
        r.vals.assign(vals, vals + 32 * k);
        for (size_t j = 0; j < k; ++j) {
            if (idx[j] > 0xffffffffull) throw InvalidArgument("update index out of range");
            if (!fr_canonical(vals + 32 * j)) throw InvalidArgument("non-canonical update value");
            r.idx[j] = (uint32_t)idx[j];
        }
        std::vector<uint32_t> sorted(r.idx);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
            throw InvalidArgument("update indices must be distinct");
        // The session's existence and size are checked under the same lock
        // that queues the request, so a concurrent close_session either sees
        // the pending request (and refuses) or runs before this check.
        std::lock_guard<std::mutex> lk(mu_);
        auto it = sessions_.find(session);
        if (it == sessions_.end()) throw InvalidArgument("unknown session");
        const uint64_t n = it->second->n;
        if (k == 0 || k > n) throw InvalidArgument("update support must hold 1..n indices");
        if (!sorted.empty() && sorted.back() >= n) throw InvalidArgument("update index out of range");
        r.ticket = next_ticket_++;
        outcomes_[r.ticket];
        queue_.push_back(std::move(r));
        cv_.notify_all();
        return queue_.back().ticket;
    }

    void wait(uint64_t ticket, uint8_t* commitment, DvgpuServeResult* res) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = outcomes_.find(ticket);
        if (it == outcomes_.end()) throw InvalidArgument("unknown ticket");
        done_cv_.wait(lk, [&] { return it->second.ready; });
        const Outcome o = it->second;
        outcomes_.erase(it);
        lk.unlock();
        if (o.status == -1) throw InvalidArgument(o.error);
        if (o.status != 0) throw CudaFailure(o.error);
        if (commitment) memcpy(commitment, o.commitment, 64);
        if (res) *res = o.res;
    }

    void set_max_batch(uint32_t m) {
        std::lock_guard<std::mutex> lk(mu_);
        max_batch_ = std::max<uint32_t>(1, m);
    }

    DvgpuServeStats stats() {
        std::lock_guard<std::mutex> lk(mu_);
        DvgpuServeStats s{};
        s.requests = stat_requests_;
        s.batches = stat_batches_;
        s.sessions = sessions_.size();
        s.resident_bytes = resident_;
        s.budget_bytes = budget_;
        s.max_batch = max_batch_;
        s.largest_batch = stat_largest_;
        s.busy_ns = stat_busy_ns_;
        s.pending = queue_.size();
        return s;
    }

private:
    // Runs fn on the engine thread and waits; exceptions come back here.
    void run(std::function<void()> fn) {
        auto task = std::make_shared<std::packaged_task<void()>>(std::move(fn));
        std::future<void> f = task->get_future();
        {
            std::lock_guard<std::mutex> lk(mu_);
            cmds_.push_back([task] { (*task)(); });
        }
        cv_.notify_all();
        f.get();
    }

    void loop() {
        cudaSetDevice(device_);
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !cmds_.empty() || !queue_.empty(); });
            if (!cmds_.empty()) {
                auto c = std::move(cmds_.front());
                cmds_.pop_front();
                lk.unlock();
                c();
                continue;
            }
            if (queue_.empty()) {
                if (stop_) break;
                continue;
            }
            // the batch: FIFO, at most one request per session
            std::vector<Request> batch;
            std::unordered_set<uint64_t> used;
            for (auto it = queue_.begin(); it != queue_.end() && batch.size() < max_batch_;) {
                if (used.count(it->session)) {
                    ++it;
                    continue;
                }
                used.insert(it->session);
                batch.push_back(std::move(*it));
                it = queue_.erase(it);
            }
            std::vector<Session*> sess;
            for (size_t r = 0; r < batch.size();) {
                auto it = sessions_.find(batch[r].session);
                if (it != sessions_.end()) {
                    sess.push_back(it->second.get());
                    ++r;
                    continue;
                }
                // cannot happen while close_session refuses sessions with
                // pending requests; fail the ticket rather than the process
                Outcome& o = outcomes_[batch[r].ticket];
                o.status = -1;
                o.error = "unknown session";
                o.ready = true;
                batch.erase(batch.begin() + r);
                done_cv_.notify_all();
            }
            if (batch.empty()) continue;
            lk.unlock();
            int status = 0;
            std::string error;
            affine_.assign(64 * batch.size(), 0);
            const uint64_t t0 = now_ns();
            dvh::XYZZ<dvh::Fq>* deltas_out = hwin_.as<dvh::XYZZ<dvh::Fq>>(batch.size());
            try {
                static_assert(sizeof(XYZZ<Fq>) == sizeof(dvh::XYZZ<dvh::Fq>), "host/device XYZZ layout");
                process(batch, sess, reinterpret_cast<uint8_t*>(deltas_out));
                // C' = C + delta C, then affine for the whole batch at once
                std::vector<dvh::XYZZ<dvh::Fq>> sums(batch.size());
                for (size_t r = 0; r < batch.size(); ++r)
                    sums[r] = dvh::xyzz_add(xyzz_of(sess[r]->commitment), deltas_out[r]);
                dvh::xyzz_batch_to_affine_bytes(sums.data(), sums.size(), affine_.data());
            } catch (const InvalidArgument& e) {
                status = -1;
                error = e.what();
            } catch (const std::exception& e) {
                status = -2;
                error = e.what();
            }
            const uint64_t t1 = now_ns();
            lk.lock();
            for (size_t r = 0; r < batch.size(); ++r) {
                Outcome& o = outcomes_[batch[r].ticket];
                o.status = status;
                o.error = error;
                if (!status) {
                    memcpy(sess[r]->commitment, &affine_[64 * r], 64);
                    memcpy(o.commitment, sess[r]->commitment, 64);
                }
                o.res.submit_ns = batch[r].submit_ns;
                o.res.start_ns = t0;
                o.res.done_ns = now_ns();
                o.res.batch_requests = (uint32_t)batch.size();
                o.res.batch_id = (uint32_t)stat_batches_;
                o.ready = true;
            }
            stat_requests_ += batch.size();
            stat_batches_++;
            stat_largest_ = std::max<uint64_t>(stat_largest_, batch.size());
            stat_busy_ns_ += t1 - t0;
            done_cv_.notify_all();
        }
        if (stream_) cudaStreamDestroy(stream_);
    }

    // One shared launch for the batch: gather + delta, then a multi-set MSM.
    void process(const std::vector<Request>& batch, const std::vector<Session*>& sess, uint8_t* deltas_out) {
        const uint32_t count = (uint32_t)batch.size();
        std::vector<uint32_t> offs(count + 1, 0);
        for (uint32_t r = 0; r < count; ++r) offs[r + 1] = offs[r] + (uint32_t)batch[r].idx.size();
        const uint32_t total = offs[count];
        // staging (one H2D copy): values (32 B each, first, so every value
        // starts on a 16-byte boundary for the 128-bit loads) | indices |
        // request offsets | base and value pointers (16-byte aligned)
        const size_t off_idx = 32ull * total;
        const size_t off_req = off_idx + 4ull * total;
        const size_t off_ptr = (off_req + 4ull * (count + 1) + 15) & ~size_t(15);
        const size_t used = off_ptr + 2 * sizeof(void*) * count;
        uint8_t* h = pinned_.as<uint8_t>(used);
        uint8_t* h_val = h;
        uint32_t* h_idx = reinterpret_cast<uint32_t*>(h + off_idx);
        uint32_t* h_off = reinterpret_cast<uint32_t*>(h + off_req);
        const G1A** h_srs = reinterpret_cast<const G1A**>(h + off_ptr);
        uint8_t** h_vals = reinterpret_cast<uint8_t**>(h + off_ptr + sizeof(void*) * count);
        for (uint32_t r = 0; r < count; ++r) {
            memcpy(h_idx + offs[r], batch[r].idx.data(), 4ull * batch[r].idx.size());
            memcpy(h_val + 32ull * offs[r], batch[r].vals.data(), batch[r].vals.size());
            h_srs[r] = sess[r]->table.view<G1A>();
            h_vals[r] = sess[r]->values.view<uint8_t>();
        }
        memcpy(h_off, offs.data(), 4ull * (count + 1));
        uint8_t* d = dstage_.as<uint8_t>(used);  // 256-byte aligned base
        DV_CUDA(cudaMemcpyAsync(d, h, used, cudaMemcpyHostToDevice, stream_));
        const uint8_t* d_val = d;
        const uint32_t* d_idx = reinterpret_cast<const uint32_t*>(d + off_idx);
        const uint32_t* d_off = reinterpret_cast<const uint32_t*>(d + off_req);
        const G1A* const* d_srs = reinterpret_cast<const G1A* const*>(d + off_ptr);
        uint8_t* const* d_vals = reinterpret_cast<uint8_t* const*>(d + off_ptr + sizeof(void*) * count);
        G1A* gathered = gathered_.as<G1A>((uint64_t)total * SERVE_W);
        uint8_t* deltas = deltas_.as<uint8_t>(32ull * total);
        const uint64_t threads = (uint64_t)total * SERVE_W;
        k_serve_prepare<<<(unsigned)((threads + 127) / 128), 128, 0, stream_>>>(total, d_off, count, d_srs, d_vals,
                                                                              d_idx, d_val, gathered, deltas);
        DV_LAUNCH();
        // one bucket set per request over the gathered window multiples
        const MsmPrecomp<Fq> pre{gathered, SERVE_C, SERVE_W};
        const MsmPlan plan = msm_plan_batch<Fq>(count, 0, total, 0, &pre);
        uint32_t* bad = err_.as<uint32_t>(1);
        DV_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), stream_));
        msm_enqueue<Fq>(ws_, nullptr, reinterpret_cast<const uint32_t*>(deltas), SetMap{d_off, nullptr, count, 0},
                        total, plan, &pre, bad, stream_);
        // the per-request sums go to the host; the engine adds them to the
        // commitments and normalises the batch with one inversion
        DV_CUDA(cudaMemcpyAsync(deltas_out, ws_.windows.view<XYZZ<Fq>>(), sizeof(XYZZ<Fq>) * count,
                                cudaMemcpyDeviceToHost, stream_));
        DV_CUDA(cudaStreamSynchronize(stream_));
        // Every fallible step is done: publish the new values.  Later
        // batches run on the same stream, so they read the committed ones.
        k_serve_commit<<<(total + 127) / 128, 128, 0, stream_>>>(total, d_off, count, d_vals, d_idx, d_val);
        DV_LAUNCH();
    }

    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    uint64_t budget_, resident_ = 0;
    uint32_t max_batch_;
    MsmWorkspace ws_;
    DevBuf stage_, err_, dstage_, gathered_, deltas_;
    PinnedBuf pinned_, hwin_;
    std::vector<uint8_t> affine_;

    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    bool stop_ = false;
    std::deque<std::function<void()>> cmds_;
    std::deque<Request> queue_;
    std::map<uint64_t, std::unique_ptr<Session>> sessions_;
    std::map<uint64_t, Outcome> outcomes_;
    uint64_t next_session_ = 1, next_ticket_ = 1;
    uint64_t stat_requests_ = 0, stat_batches_ = 0, stat_largest_ = 0, stat_busy_ns_ = 0;
    std::thread worker_;
};

int fail_text(int status, const std::string& msg, char* error, size_t cap) {
    if (error && cap) {
        const size_t k = std::min(cap - 1, msg.size());
        memcpy(error, msg.data(), k);
        error[k] = '\0';
    }
    return status;
}

template <class Fn>
int serve_guard(char* error, size_t cap, Fn&& fn) {
    try {
        fn();
        return 0;
    } catch (const InvalidArgument& e) {
        return fail_text(-1, e.what(), error, cap);
    } catch (const std::exception& e) {
        return fail_text(-2, e.what(), error, cap);
    } catch (...) {
        return fail_text(-3, "unknown native exception", error, cap);
    }
}

}  // namespace
}  // namespace dv

using dv::Server;

extern "C" int dvgpu_serve_create(uint64_t hbm_budget_bytes, uint32_t max_batch, void** server, char* error,
                                  size_t cap) {
    return dv::serve_guard(error, cap, [&] {
        if (!server) throw dv::InvalidArgument("null server output");
        *server = nullptr;
        // the calling thread's current device (one server per GPU, e.g. one per rank)
        *server = new Server(hbm_budget_bytes, max_batch);
    });
}

extern "C" void dvgpu_serve_destroy(void* server) { delete static_cast<Server*>(server); }

extern "C" int dvgpu_serve_open_session(void* server, const uint8_t* srs_g1, const uint8_t* values, size_t n,
                                        uint64_t* session, uint8_t* commitment, char* error, size_t cap) {
    return dv::serve_guard(error, cap, [&] {
        if (!server || !srs_g1 || !values || !session || !commitment || n == 0 || n > DVGPU_MAX_MSM_SIZE)
            throw dv::InvalidArgument("invalid session arguments");
        *session = static_cast<Server*>(server)->open_session(srs_g1, values, n, commitment);
    });
}

extern "C" int dvgpu_serve_close_session(void* server, uint64_t session, char* error, size_t cap) {
    return dv::serve_guard(error, cap, [&] {
        if (!server) throw dv::InvalidArgument("null server");
        static_cast<Server*>(server)->close_session(session);
    });
}

extern "C" int dvgpu_serve_submit(void* server, uint64_t session, const uint64_t* indices, const uint8_t* values,
                                  size_t k, uint64_t* ticket, char* error, size_t cap) {
    return dv::serve_guard(error, cap, [&] {
        if (!server || !ticket || (k && (!indices || !values))) throw dv::InvalidArgument("invalid update arguments");
        *ticket = static_cast<Server*>(server)->submit(session, indices, values, k);
    });
}

extern "C" int dvgpu_serve_wait(void* server, uint64_t ticket, uint8_t* commitment, DvgpuServeResult* result,
                                char* error, size_t cap) {
    return dv::serve_guard(error, cap, [&] {
        if (!server) throw dv::InvalidArgument("null server");
        static_cast<Server*>(server)->wait(ticket, commitment, result);
    });
}

extern "C" int dvgpu_serve_set_max_batch(void* server, uint32_t max_batch) {
    if (!server) return -1;
    static_cast<Server*>(server)->set_max_batch(max_batch);
    return 0;
}

extern "C" int dvgpu_serve_stats(void* server, DvgpuServeStats* out) {
    if (!server || !out) return -1;
    *out = static_cast<Server*>(server)->stats();
    return 0;
}
