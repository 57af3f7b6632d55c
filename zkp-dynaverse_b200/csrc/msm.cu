// Pippenger MSM kernels and their launch sequence (see msm.cuh).
#include <algorithm>
#include <cstring>
#include <vector>

#include "host_curve.hpp"
#include "msm.cuh"

namespace dv {

namespace {

constexpr uint32_t NO_INDEX = 0xffffffffu;

DV_INL uint32_t window_raw(const uint32_t* s, int bit, int c) {
    if (bit >= 256) return 0;
    const int limb = bit >> 5, sh = bit & 31;
    uint32_t v = s[limb] >> sh;
    if (sh + c > 32 && limb + 1 < 8) v |= s[limb + 1] << (32 - sh);
    return v & ((1u << c) - 1u);
}

DV_INL void load_scalar(const uint32_t* scalars, uint32_t i, uint32_t* s) {
    const uint4* q = reinterpret_cast<const uint4*>(scalars + 8ull * i);
    const uint4 a = q[0], b = q[1];
    s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
    s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
}

DV_INL uint32_t set_of(const uint32_t* set_off, uint32_t count, uint32_t i) {
    // largest k with set_off[k] <= i
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (set_off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// 1. Histogram of signed digits.
__global__ void k_hist(const uint32_t* __restrict__ scalars, uint32_t n, const uint32_t* __restrict__ set_off,
                       uint32_t count, int c, int W, uint32_t* __restrict__ counts, uint32_t* __restrict__ first_bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s[8];
    load_scalar(scalars, i, s);
    if (!Fr::is_canonical(s)) {
        atomicMin(first_bad, i);
        return;
    }
    const uint32_t set = count > 1 ? set_of(set_off, count, i) : 0;
    const uint32_t B = 1u << (c - 1), full = 1u << c;
    uint32_t* base = counts + (size_t)set * W * B;
    uint32_t carry = 0;
    for (int w = 0; w < W; ++w) {
        const uint32_t d = window_raw(s, w * c, c) + carry;
        const bool neg = d > B;
        const uint32_t mag = neg ? full - d : d;
        carry = neg ? 1u : 0u;
        if (mag) atomicAdd(base + (size_t)w * B + mag - 1, 1u);
    }
}

// 2. Exclusive scan of counts (one block of 1024 threads).
__global__ void __launch_bounds__(1024) k_scan(const uint32_t* __restrict__ counts, uint32_t nb,
                                               uint32_t* __restrict__ offsets, uint32_t* __restrict__ cursor) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (nb + 1023) / 1024;
    const uint32_t lo = min(nb, t * per), hi = min(nb, lo + per);
    uint32_t local = 0;
    for (uint32_t i = lo; i < hi; ++i) local += counts[i];
    part[t] = local;
    __syncthreads();
    for (uint32_t d = 1; d < 1024; d <<= 1) {
        const uint32_t v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - local;  // exclusive prefix
    for (uint32_t i = lo; i < hi; ++i) {
        offsets[i] = run;
        cursor[i] = run;
        run += counts[i];
    }
    if (t == 1023) offsets[nb] = part[1023];
}

// 3. Scatter (point index | sign << 31) into bucket order.
__global__ void k_scatter(const uint32_t* __restrict__ scalars, uint32_t n, const uint32_t* __restrict__ set_off,
                          uint32_t count, int c, int W, uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s[8];
    load_scalar(scalars, i, s);
    if (!Fr::is_canonical(s)) return;
    const uint32_t set = count > 1 ? set_of(set_off, count, i) : 0;
    const uint32_t B = 1u << (c - 1), full = 1u << c;
    uint32_t* base = cursor + (size_t)set * W * B;
    uint32_t carry = 0;
    for (int w = 0; w < W; ++w) {
        const uint32_t d = window_raw(s, w * c, c) + carry;
        const bool neg = d > B;
        const uint32_t mag = neg ? full - d : d;
        carry = neg ? 1u : 0u;
        if (mag) {
            const uint32_t pos = atomicAdd(base + (size_t)w * B + mag - 1, 1u);
            sorted[pos] = i | (neg ? 0x80000000u : 0u);
        }
    }
}

// 4. Balanced accumulation over the sorted list.
template <class F>
__global__ void __launch_bounds__(128) k_accum(const Affine<F>* __restrict__ pts, const uint32_t* __restrict__ sorted,
                                               const uint32_t* __restrict__ offsets, uint32_t nb,
                                               XYZZ<F>* __restrict__ buckets, int* __restrict__ pgid,
                                               XYZZ<F>* __restrict__ ppt) {
    const uint32_t T = gridDim.x * blockDim.x;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t M = offsets[nb];
    const uint32_t L = (M + T - 1) / T;
    int head_gid = -1, tail_gid = -1;
    XYZZ<F> head = XYZZ<F>::inf(), tail = XYZZ<F>::inf();
    const uint64_t start64 = (uint64_t)t * L;
    if (L && start64 < M) {
        const uint32_t start = (uint32_t)start64;
        const uint32_t end = min(M, start + L);
        uint32_t lo = 0, hi = nb;  // offsets[lo] <= start < offsets[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= start) lo = mid; else hi = mid;
        }
        uint32_t g = lo;
        uint32_t gbeg = offsets[g], gend = offsets[g + 1];
        XYZZ<F> acc = XYZZ<F>::inf();
        uint32_t run_start = start;
        for (uint32_t pos = start; pos < end; ++pos) {
            if (pos == gend) {
                // bucket g ended inside this slice: run [run_start, pos)
                if (gbeg < run_start) { head_gid = (int)g; head = acc; }
                else buckets[g] = acc;
                do { ++g; gbeg = gend; gend = offsets[g + 1]; } while (gend <= pos);
                acc = XYZZ<F>::inf();
                run_start = pos;
            }
            const uint32_t e = sorted[pos];
            Affine<F> p = pts[e & 0x7fffffffu];
            if (e >> 31) p.y = F::neg(p.y);
            acc = XYZZ<F>::add_affine(acc, p);
        }
        const bool before = gbeg < run_start;
        const bool after = gend > end;
        if (before) { head_gid = (int)g; head = acc; }
        else if (after) { tail_gid = (int)g; tail = acc; }
        else buckets[g] = acc;
    }
    pgid[2 * t] = head_gid;
    pgid[2 * t + 1] = tail_gid;
    ppt[2 * t] = head;
    ppt[2 * t + 1] = tail;
}

// 5. Merge partials of buckets that span slices.  The owner of bucket g is
// the slice whose tail holds g; the following slices hold g in their heads.
template <class F>
__global__ void k_fixup(const int* __restrict__ pgid, const XYZZ<F>* __restrict__ ppt, uint32_t T,
                        XYZZ<F>* __restrict__ buckets) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int g = pgid[2 * t + 1];
    if (g < 0) return;
    XYZZ<F> acc = ppt[2 * t + 1];
    for (uint32_t k = t + 1; k < T && pgid[2 * k] == g; ++k) acc = XYZZ<F>::add(acc, ppt[2 * k]);
    buckets[g] = acc;
}

// 6. Segment values: for segment j of window (set, w), with buckets
// b in [j s, (j+1) s) weighted by (b + 1):
//   V_j = sum_b (b - j s + 1) B_b  +  (j s) * sum_b B_b
template <class F>
__global__ void __launch_bounds__(128) k_segments(const XYZZ<F>* __restrict__ buckets, const uint32_t* __restrict__ offsets,
                                                  uint32_t B, uint32_t NW, int seg_log, XYZZ<F>* __restrict__ segs) {
    const uint32_t S = B >> seg_log;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= NW * S) return;
    const uint32_t w = tid / S, j = tid % S;
    const uint32_t s = 1u << seg_log;
    XYZZ<F> R = XYZZ<F>::inf(), Tsum = XYZZ<F>::inf();
    const size_t base = (size_t)w * B + (size_t)j * s;
    for (int b = (int)s - 1; b >= 0; --b) {
        const size_t g = base + b;
        if (offsets[g + 1] != offsets[g]) R = XYZZ<F>::add(R, buckets[g]);
        Tsum = XYZZ<F>::add(Tsum, R);
    }
    // (j s) * R = (j * R) doubled seg_log times
    XYZZ<F> jr = XYZZ<F>::inf();
    if (j && !R.is_inf()) {
        const int top = 31 - __clz(j);
        for (int bit = top; bit >= 0; --bit) {
            jr = XYZZ<F>::dbl(jr);
            if ((j >> bit) & 1) jr = XYZZ<F>::add(jr, R);
        }
        for (int k = 0; k < seg_log; ++k) jr = XYZZ<F>::dbl(jr);
    }
    segs[tid] = XYZZ<F>::add(Tsum, jr);
}

// 7. Sum of the S segment values of each (set, window): one block each.
template <class F, int THREADS>
__global__ void __launch_bounds__(THREADS) k_wsum(const XYZZ<F>* __restrict__ segs, uint32_t S,
                                                  XYZZ<F>* __restrict__ out) {
    __shared__ XYZZ<F> sh[THREADS];
    const uint32_t w = blockIdx.x, t = threadIdx.x;
    XYZZ<F> acc = XYZZ<F>::inf();
    for (uint32_t j = t; j < S; j += THREADS) acc = XYZZ<F>::add(acc, segs[(size_t)w * S + j]);
    sh[t] = acc;
    __syncthreads();
    for (int d = THREADS / 2; d > 0; d >>= 1) {
        if ((int)t < d) sh[t] = XYZZ<F>::add(sh[t], sh[t + d]);
        __syncthreads();
    }
    if (t == 0) out[w] = sh[0];
}

// Canonical -> Montgomery conversion with validation.
DV_INL bool all_zero_words(const uint32_t* w, int n) {
    uint32_t x = 0;
    for (int i = 0; i < n; ++i) x |= w[i];
    return x == 0;
}

__global__ void k_convert_g1(const uint8_t* __restrict__ canon, G1A* __restrict__ out, uint64_t n,
                             uint32_t* __restrict__ first_bad) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t x[8], y[8];
    load_words(canon + 64 * i, x);
    load_words(canon + 64 * i + 32, y);
    G1A p;
    if (all_zero_words(x, 8) && all_zero_words(y, 8)) {
        p = G1A::inf();
    } else {
        if (!Fq::is_canonical(x) || !Fq::is_canonical(y)) { atomicMin(first_bad, (uint32_t)i); return; }
        p.x = Fq::from_canonical(x);
        p.y = Fq::from_canonical(y);
        if (!CurveOps<Fq>::on_curve(p)) { atomicMin(first_bad, (uint32_t)i); return; }
    }
    out[i] = p;
}

__global__ void k_convert_g2(const uint8_t* __restrict__ canon, G2A* __restrict__ out, uint64_t n,
                             uint32_t* __restrict__ first_bad) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t w[4][8];
    bool zero = true;
    for (int j = 0; j < 4; ++j) {
        load_words(canon + 128 * i + 32 * j, w[j]);
        zero &= all_zero_words(w[j], 8);
    }
    G2A p;
    if (zero) {
        p = G2A::inf();
    } else {
        for (int j = 0; j < 4; ++j)
            if (!Fq::is_canonical(w[j])) { atomicMin(first_bad, (uint32_t)i); return; }
        p.x = {Fq::from_canonical(w[0]), Fq::from_canonical(w[1])};
        p.y = {Fq::from_canonical(w[2]), Fq::from_canonical(w[3])};
        if (!CurveOps<Fq2>::on_curve(p)) { atomicMin(first_bad, (uint32_t)i); return; }
    }
    out[i] = p;
}

template <class F>
__global__ void k_gather(const Affine<F>* __restrict__ bases, uint64_t nbases, const uint64_t* __restrict__ idx,
                         uint64_t k, Affine<F>* __restrict__ out, uint32_t* __restrict__ first_bad) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const uint64_t i = idx[j];
    if (i >= nbases) { atomicMin(first_bad, (uint32_t)j); return; }
    out[j] = bases[i];
}

inline unsigned blocks_for(uint64_t n, unsigned threads) { return (unsigned)((n + threads - 1) / threads); }

// Host Horner over windows: sum_w 2^(c w) S_w.
template <class HF>
void horner(const dvh::XYZZ<HF>* win, int W, int c, uint8_t* out) {
    dvh::XYZZ<HF> acc = dvh::xyzz_inf<HF>();
    for (int w = W - 1; w >= 0; --w) {
        for (int k = 0; k < c; ++k) acc = dvh::xyzz_dbl(acc);
        acc = dvh::xyzz_add(acc, win[w]);
    }
    dvh::xyzz_to_affine_bytes(acc, out);
}

template <class F>
struct HostOf;
template <>
struct HostOf<Fq> { typedef dvh::Fq T; };
template <>
struct HostOf<Fq2> { typedef dvh::Fq2 T; };

}  // namespace

MsmPlan msm_plan(uint64_t n, int force_c) {
    MsmPlan p;
    int best_c = 4;
    double best = 1e300;
    for (int c = 4; c <= 20; ++c) {
        const double W = (255 + c - 1) / c;
        const double cost = W * (10.0 * (double)n + 28.0 * (double)(1u << (c - 1)));
        if (cost < best) { best = cost; best_c = c; }
    }
    p.c = force_c ? force_c : best_c;
    p.windows = (255 + p.c - 1) / p.c;
    p.buckets = 1u << (p.c - 1);
    p.seg_log = std::min(4, p.c - 1);
    return p;
}

template <class F>
void convert_points(const uint8_t* d_canon, Affine<F>* d_out, uint64_t n, uint32_t* d_first_bad, cudaStream_t st) {
    if (!n) return;
    if constexpr (sizeof(F) == sizeof(Fq)) k_convert_g1<<<blocks_for(n, 128), 128, 0, st>>>(d_canon, d_out, n, d_first_bad);
    else k_convert_g2<<<blocks_for(n, 128), 128, 0, st>>>(d_canon, d_out, n, d_first_bad);
    DV_LAUNCH();
}

template <class F>
void gather_points(const Affine<F>* d_bases, uint64_t nbases, const uint64_t* d_idx, uint64_t k, Affine<F>* d_out,
                   uint32_t* d_first_bad, cudaStream_t st) {
    if (!k) return;
    k_gather<F><<<blocks_for(k, 256), 256, 0, st>>>(d_bases, nbases, d_idx, k, d_out, d_first_bad);
    DV_LAUNCH();
}

template <class F>
void msm_run(MsmWorkspace& ws, const Affine<F>* d_points, const uint32_t* d_scalars, const uint32_t* set_offsets,
             uint32_t count, int force_c, cudaStream_t st, uint8_t* host_out, MsmStats* stats) {
    typedef typename HostOf<F>::T HF;
    const size_t out_bytes = 2 * sizeof(F);
    const uint32_t n = set_offsets[count];
    uint32_t max_set = 0;
    for (uint32_t k = 0; k < count; ++k) max_set = std::max(max_set, set_offsets[k + 1] - set_offsets[k]);
    if (n == 0 || count == 0) {
        memset(host_out, 0, (size_t)count * out_bytes);
        return;
    }
    MsmPlan plan = msm_plan(max_set, force_c);
    // Bound the bucket table of a batch: count * windows * buckets <= 2^26
    // (8 GB of G1 XYZZ buckets); smaller windows trade buckets for windows.
    while (plan.c > 4 && (uint64_t)count * plan.windows * plan.buckets > (1ull << 26)) {
        plan.c--;
        plan.windows = (255 + plan.c - 1) / plan.c;
        plan.buckets = 1u << (plan.c - 1);
        plan.seg_log = std::min(4, plan.c - 1);
    }
    if ((uint64_t)count * plan.windows * plan.buckets > (1ull << 31) || (uint64_t)n * plan.windows > 0xffffffffull)
        throw InvalidArgument("MSM batch too large for one launch sequence");
    const int c = plan.c, W = plan.windows;
    const uint32_t B = plan.buckets;
    const uint32_t NW = count * (uint32_t)W;
    const uint32_t NB = NW * B;

    uint32_t* d_set = ws.set_off.as<uint32_t>(count + 1);
    uint32_t* d_counts = ws.counts.as<uint32_t>(NB);
    uint32_t* d_offsets = ws.offsets.as<uint32_t>(NB + 1);
    uint32_t* d_cursor = ws.cursor.as<uint32_t>(NB);
    uint32_t* d_sorted = ws.sorted.as<uint32_t>((size_t)n * W);
    XYZZ<F>* d_buckets = ws.buckets.as<XYZZ<F>>(NB);
    uint32_t* d_err = ws.err.as<uint32_t>(1);
    uint32_t* h_err = ws.host_err.as<uint32_t>(1);

    DV_CUDA(cudaMemcpyAsync(d_set, set_offsets, (count + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)NB * sizeof(uint32_t), st));
    DV_CUDA(cudaMemsetAsync(d_err, 0xff, sizeof(uint32_t), st));

    MsmTimeline& tl = ws.timeline;
    auto mark = [&](int k) {
        if (tl.enabled) DV_CUDA(cudaEventRecord(tl.ev[k], st));
    };
    mark(0);
    k_hist<<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, d_set, count, c, W, d_counts, d_err);
    DV_LAUNCH();
    mark(1);
    k_scan<<<1, 1024, 0, st>>>(d_counts, NB, d_offsets, d_cursor);
    DV_LAUNCH();
    mark(2);
    k_scatter<<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, d_set, count, c, W, d_cursor, d_sorted);
    DV_LAUNCH();
    mark(3);

    int per_sm = 0;
    DV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_accum<F>, 128, 0));
    per_sm = std::max(1, per_sm);
    const uint64_t max_entries = (uint64_t)n * W;
    uint32_t grid = (uint32_t)sm_count() * (uint32_t)per_sm;
    // small inputs: keep at least ~8 entries per thread
    grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(grid, (max_entries + 8 * 128 - 1) / (8 * 128)));
    const uint32_t T = grid * 128;
    int* d_pgid = ws.pgid.as<int>(2ull * T);
    XYZZ<F>* d_ppt = ws.ppt.as<XYZZ<F>>(2ull * T);
    k_accum<F><<<grid, 128, 0, st>>>(d_points, d_sorted, d_offsets, NB, d_buckets, d_pgid, d_ppt);
    DV_LAUNCH();
    mark(4);
    k_fixup<F><<<blocks_for(T, 128), 128, 0, st>>>(d_pgid, d_ppt, T, d_buckets);
    DV_LAUNCH();
    mark(5);

    const int seg_log = plan.seg_log;
    const uint32_t S = B >> seg_log;
    XYZZ<F>* d_segs = ws.segs.as<XYZZ<F>>((size_t)NW * S);
    XYZZ<F>* d_win = ws.windows.as<XYZZ<F>>(NW);
    k_segments<F><<<blocks_for((uint64_t)NW * S, 128), 128, 0, st>>>(d_buckets, d_offsets, B, NW, seg_log, d_segs);
    DV_LAUNCH();
    mark(6);
    k_wsum<F, 128><<<NW, 128, 0, st>>>(d_segs, S, d_win);
    DV_LAUNCH();
    mark(7);

    XYZZ<F>* h_win = ws.host_windows.as<XYZZ<F>>(NW);
    DV_CUDA(cudaMemcpyAsync(h_win, d_win, (size_t)NW * sizeof(XYZZ<F>), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(h_err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (*h_err != NO_INDEX)
        throw InvalidArgument("non-canonical scalar at index " + std::to_string(*h_err));
    static_assert(sizeof(XYZZ<F>) == sizeof(dvh::XYZZ<HF>), "host/device XYZZ layout");
    const auto* hw = reinterpret_cast<const dvh::XYZZ<HF>*>(h_win);
    for (uint32_t k = 0; k < count; ++k) horner(hw + (size_t)k * W, W, c, host_out + (size_t)k * out_bytes);
    if (tl.enabled) {
        DV_CUDA(cudaEventRecord(tl.ev[8], st));
        DV_CUDA(cudaEventSynchronize(tl.ev[8]));
        for (int k = 0; k < MSM_PHASES; ++k) {
            float ms = 0;
            DV_CUDA(cudaEventElapsedTime(&ms, tl.ev[k], tl.ev[k + 1]));
            tl.ms[k] += ms;
        }
        tl.calls++;
        tl.accum_mixed_adds += (uint64_t)n * W;
    }
    if (stats) {
        stats->calls++;
        stats->sets += count;
        stats->points += n;
        stats->last_c = (uint64_t)c;
    }
}

template void msm_run<Fq>(MsmWorkspace&, const Affine<Fq>*, const uint32_t*, const uint32_t*, uint32_t, int,
                          cudaStream_t, uint8_t*, MsmStats*);
template void msm_run<Fq2>(MsmWorkspace&, const Affine<Fq2>*, const uint32_t*, const uint32_t*, uint32_t, int,
                           cudaStream_t, uint8_t*, MsmStats*);
template void convert_points<Fq>(const uint8_t*, Affine<Fq>*, uint64_t, uint32_t*, cudaStream_t);
template void convert_points<Fq2>(const uint8_t*, Affine<Fq2>*, uint64_t, uint32_t*, cudaStream_t);
template void gather_points<Fq>(const Affine<Fq>*, uint64_t, const uint64_t*, uint64_t, Affine<Fq>*, uint32_t*,
                                cudaStream_t);
template void gather_points<Fq2>(const Affine<Fq2>*, uint64_t, const uint64_t*, uint64_t, Affine<Fq2>*, uint32_t*,
                                 cudaStream_t);

}  // namespace dv
