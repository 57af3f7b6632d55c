// Pippenger MSM kernels and their launch sequence (see msm.cuh).
#include <algorithm>
#include <cstring>
#include <vector>

#include "host_curve.hpp"
#include "msm.cuh"

namespace dv {

namespace {

constexpr uint32_t NO_INDEX = 0xffffffffu;

// Bucket-reduction segment length 2^DV_SEG_LOG (buckets per thread in the
// first level; doubled for long G1 windows).
#ifndef DV_SEG_LOG
#define DV_SEG_LOG 3
#endif

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

// Where digit i of a launch comes from: its set, its scalar and its point.
DV_INL void locate(const SetMap& m, uint32_t i, uint32_t& set, uint32_t& sidx, uint32_t& pidx) {
    set = m.count > 1 ? set_of(m.off, m.count, i) : 0;
    const uint32_t rel = i - (m.count > 1 ? m.off[set] : 0u);
    sidx = m.term_scalar ? m.term_scalar[i] : m.src ? m.src[set] + rel : i;
    pidx = m.term_point ? m.term_point[i] : m.prefix ? rel : sidx;
}

// 1. Histogram of signed digits.
template <bool PRE>
__global__ void k_hist(const uint32_t* __restrict__ scalars, uint32_t n, const SetMap m, int c, int W,
                       uint32_t* __restrict__ counts, uint32_t* __restrict__ first_bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t set, sidx, pidx;
    locate(m, i, set, sidx, pidx);
    uint32_t s[8];
    load_scalar(scalars, sidx, s);
    if (!Fr::is_canonical(s)) {
        atomicMin(first_bad, sidx);
        return;
    }
    const uint32_t B = 1u << (c - 1), full = 1u << c;
    // PRE: precomputed window multiples share one bucket set per MSM
    const uint32_t base = PRE ? set * B : set * (uint32_t)W * B;
    const uint32_t active = __activemask();
    const uint32_t lane = threadIdx.x & 31;
    uint32_t carry = 0;
    for (int w = 0; w < W; ++w) {
        const uint32_t d = window_raw(s, w * c, c) + carry;
        const bool neg = d > B;
        const uint32_t mag = neg ? full - d : d;
        carry = neg ? 1u : 0u;
        // Warp-aggregated increment: lanes hitting the same bucket (skewed
        // digits, e.g. a top window with few bits) issue one atomic.
        const uint32_t key = mag ? base + (PRE ? 0u : (uint32_t)w * B) + mag - 1 : NO_INDEX;
        const uint32_t peers = __match_any_sync(active, key);
        if (key != NO_INDEX && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(counts + key, (uint32_t)__popc(peers));
    }
}

// 2. Exclusive scan of the counts: tiles of 4096 (1024 threads x 4), three
// passes -- tile sums, scan of the tile sums, per-tile scan with its prefix.
constexpr uint32_t SCAN_TILE = 4096;

// Exclusive scan of one value per thread over a 1024-thread block.
DV_INL uint32_t block_exclusive_scan(uint32_t v, uint32_t* block_total) {
    __shared__ uint32_t warp_sums[32];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = warp_sums[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= (uint32_t)d) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t prefix = (wid ? warp_sums[wid - 1] : 0u) + x - v;
    if (block_total) *block_total = warp_sums[31];
    __syncthreads();
    return prefix;
}

DV_INL void load4(const uint32_t* counts, uint32_t nb, uint32_t i, uint32_t* v) {
    if (i + 3 < nb) {
        const uint4 q = *reinterpret_cast<const uint4*>(counts + i);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
        for (int k = 0; k < 4; ++k) v[k] = i + k < nb ? counts[i + k] : 0u;
    }
}

__global__ void __launch_bounds__(1024) k_scan_tiles(const uint32_t* __restrict__ counts, uint32_t nb,
                                                     uint32_t* __restrict__ tile_sums) {
    const uint32_t i = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
    uint32_t v[4];
    load4(counts, nb, i, v);
    uint32_t total;
    block_exclusive_scan(v[0] + v[1] + v[2] + v[3], &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_top(uint32_t* __restrict__ tile_sums, uint32_t ntiles,
                                                   uint32_t* __restrict__ grand_total) {
    const uint32_t per = (ntiles + 1023) / 1024;
    const uint32_t lo = min(ntiles, threadIdx.x * per), hi = min(ntiles, lo + per);
    uint32_t local = 0;
    for (uint32_t i = lo; i < hi; ++i) local += tile_sums[i];
    uint32_t total;
    uint32_t run = block_exclusive_scan(local, &total);
    for (uint32_t i = lo; i < hi; ++i) {
        const uint32_t v = tile_sums[i];
        tile_sums[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) *grand_total = total;
}

__global__ void __launch_bounds__(1024) k_scan_apply(const uint32_t* __restrict__ counts, uint32_t nb,
                                                     const uint32_t* __restrict__ tile_prefix,
                                                     uint32_t* __restrict__ offsets, uint32_t* __restrict__ cursor) {
    const uint32_t i = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
    uint32_t v[4];
    load4(counts, nb, i, v);
    uint32_t run = tile_prefix[blockIdx.x] + block_exclusive_scan(v[0] + v[1] + v[2] + v[3], nullptr);
    for (int k = 0; k < 4; ++k) {
        if (i + k < nb) {
            offsets[i + k] = run;
            cursor[i + k] = run;
        }
        run += v[k];
    }
}

// 3. Scatter (point index | sign << 31) into bucket order.
template <bool PRE>
__global__ void k_scatter(const uint32_t* __restrict__ scalars, uint32_t n, const SetMap m, int c, int W,
                          uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t set, sidx, pidx;
    locate(m, i, set, sidx, pidx);
    uint32_t s[8];
    load_scalar(scalars, sidx, s);
    if (!Fr::is_canonical(s)) return;
    const uint32_t B = 1u << (c - 1), full = 1u << c;
    // PRE: precomputed window multiples share one bucket set per MSM
    const uint32_t base = PRE ? set * B : set * (uint32_t)W * B;
    const uint32_t active = __activemask();
    const uint32_t lane = threadIdx.x & 31;
    uint32_t carry = 0;
    for (int w = 0; w < W; ++w) {
        const uint32_t d = window_raw(s, w * c, c) + carry;
        const bool neg = d > B;
        const uint32_t mag = neg ? full - d : d;
        carry = neg ? 1u : 0u;
        const uint32_t key = mag ? base + (PRE ? 0u : (uint32_t)w * B) + mag - 1 : NO_INDEX;
        const uint32_t peers = __match_any_sync(active, key);
        if (key != NO_INDEX) {
            // one atomic per group of lanes with the same bucket; each lane
            // takes its rank within the group
            const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
            uint32_t pos = 0;
            if (lane == leader) pos = atomicAdd(cursor + key, (uint32_t)__popc(peers));
            pos = __shfl_sync(peers, pos, leader) + (uint32_t)__popc(peers & ((1u << lane) - 1u));
            const uint32_t idx = PRE ? pidx * (uint32_t)W + (uint32_t)w : pidx;  // PRE: table entry 2^(c w) P_i
            sorted[pos] = idx | (neg ? 0x80000000u : 0u);
        }
    }
}

// 4. Balanced accumulation over the sorted list.
#ifndef DV_ACCUM_MINB
#define DV_ACCUM_MINB 4
#endif
template <class F>
__global__ void __launch_bounds__(128, DV_ACCUM_MINB) k_accum(const Affine<F>* __restrict__ pts, const uint32_t* __restrict__ sorted,
                                               const uint32_t* __restrict__ offsets, uint32_t nb,
                                               XYZZ<F>* __restrict__ buckets, int* __restrict__ pgid,
                                               XYZZ<F>* __restrict__ ppt) {
    // buckets [0, nb) of this launch cover sorted positions [offsets[0], offsets[nb])
    const uint32_t T = gridDim.x * blockDim.x;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t M0 = offsets[0];
    const uint32_t M = offsets[nb] - M0;
    const uint32_t L = (M + T - 1) / T;
    int head_gid = -1, tail_gid = -1;
    XYZZ<F> head = XYZZ<F>::inf(), tail = XYZZ<F>::inf();
    const uint64_t rel64 = (uint64_t)t * L;
    if (L && rel64 < M) {
        const uint32_t start = M0 + (uint32_t)rel64;
        const uint32_t end = M0 + min(M, (uint32_t)rel64 + L);
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
// Chains of more than FIX_SHORT heads (a bucket spanning many slices: skewed
// digits) are queued for k_fixup_long, which merges them with a block-wide
// tree instead of one serial walk.
constexpr uint32_t FIX_SHORT = 32;

template <class F>
__global__ void k_fixup(const int* __restrict__ pgid, const XYZZ<F>* __restrict__ ppt, uint32_t T,
                        XYZZ<F>* __restrict__ buckets, uint32_t* __restrict__ long_list,
                        uint32_t* __restrict__ long_count) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int g = pgid[2 * t + 1];
    if (g < 0) return;
    uint32_t end = t + 1;
    while (end < T && pgid[2 * end] == g && end - t <= FIX_SHORT) ++end;
    if (end < T && pgid[2 * end] == g) {
        long_list[atomicAdd(long_count, 1u)] = t;
        return;
    }
    XYZZ<F> acc = ppt[2 * t + 1];
    for (uint32_t k = t + 1; k < end; ++k) acc = XYZZ<F>::add(acc, ppt[2 * k]);
    buckets[g] = acc;
}

template <class F, int TH>
__global__ void __launch_bounds__(TH) k_fixup_long(const int* __restrict__ pgid, const XYZZ<F>* __restrict__ ppt,
                                                   uint32_t T, XYZZ<F>* __restrict__ buckets,
                                                   const uint32_t* __restrict__ long_list,
                                                   const uint32_t* __restrict__ long_count) {
    __shared__ XYZZ<F> sh[TH];
    const uint32_t nlong = *long_count;
    for (uint32_t item = blockIdx.x; item < nlong; item += gridDim.x) {
        const uint32_t t0 = long_list[item];
        const int g = pgid[2 * t0 + 1];
        XYZZ<F> acc = threadIdx.x == 0 ? ppt[2 * t0 + 1] : XYZZ<F>::inf();
        // the heads of g are contiguous from t0 + 1: stop at the first other key
        for (uint32_t k = t0 + 1 + threadIdx.x; k < T && pgid[2 * k] == g; k += TH)
            acc = XYZZ<F>::add(acc, ppt[2 * k]);
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int d = TH / 2; d > 0; d >>= 1) {
            if ((int)threadIdx.x < d) sh[threadIdx.x] = XYZZ<F>::add(sh[threadIdx.x], sh[threadIdx.x + d]);
            __syncthreads();
        }
        if (threadIdx.x == 0) buckets[g] = sh[0];
        __syncthreads();
    }
}

// 6. Bucket reduction.  Window (set, w) needs
//      S_w = sum_b (b + 1) B_b,   b < 2^(c-1).
// Every level carries a window as pairs (U_j, V_j) with
//      S_w = sum_j U_j + sum_j j V_j ,
// V_j already multiplied by the weight unit of its level.  Level 1:
// segment j holds buckets [j s, (j+1) s); a running sum from the top gives
//      U_j = sum_i (i + 1) B_{js+i},   V_j = s sum_i B_{js+i}.
// Grouping G consecutive pairs (j = G q + l) gives the next level:
//      U'_q = sum_l U_{Gq+l} + sum_l l V_{Gq+l} = sum_l (U_l + Suf_{l+1}),
//      V'_q = G sum_l V_{Gq+l},
// with Suf the group's suffix sums of V; the doublings for G apply to one
// sum per group, so the critical path holds log2(total weight) of them.

// Additions and doublings of the reduction: few threads per bucket set on a
// dependent chain, so over Fq the products go out in pairs.
template <class F>
DV_INL XYZZ<F> wadd(const XYZZ<F>& p, const XYZZ<F>& q) {
    if constexpr (sizeof(F) == sizeof(Fq)) return XYZZ<F>::add_paired(p, q);
    else return XYZZ<F>::add(p, q);
}
template <class F>
DV_INL XYZZ<F> wdbl(const XYZZ<F>& p) {
    if constexpr (sizeof(F) == sizeof(Fq)) return XYZZ<F>::dbl_paired(p);
    else return XYZZ<F>::dbl(p);
}
template <class F>
DV_INL XYZZ<F> shfl_down_xyzz(const XYZZ<F>& p, int d) {
    return {shfl_down(p.x, d), shfl_down(p.y, d), shfl_down(p.zz, d), shfl_down(p.zzz, d)};
}
template <class F>
DV_INL XYZZ<F> shfl_idx_xyzz(const XYZZ<F>& p, int l) {
    return {shfl_idx(p.x, l), shfl_idx(p.y, l), shfl_idx(p.zz, l), shfl_idx(p.zzz, l)};
}

// Level 1: one segment of s buckets per thread.
template <class F>
__global__ void __launch_bounds__(128) k_segments(const XYZZ<F>* __restrict__ buckets, const uint32_t* __restrict__ offsets,
                                                  uint32_t B, uint32_t NW, int seg_log, XYZZ<F>* __restrict__ seg_u,
                                                  XYZZ<F>* __restrict__ seg_v) {
    const uint32_t S = B >> seg_log;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= NW * S) return;
    const uint32_t w = tid / S, j = tid % S;
    const uint32_t s = 1u << seg_log;
    XYZZ<F> R = XYZZ<F>::inf(), U = XYZZ<F>::inf();
    const size_t base = (size_t)w * B + (size_t)j * s;
    for (int b = (int)s - 1; b >= 0; --b) {
        const size_t g = base + b;
        if (offsets[g + 1] != offsets[g]) R = wadd<F>(R, buckets[g]);
        U = wadd<F>(U, R);
    }
    for (int i = 0; i < seg_log; ++i) R = wdbl<F>(R);  // V = s R
    seg_u[tid] = U;
    seg_v[tid] = R;
}

// Upper levels: blocks of P pairs (G = P), windows of S pairs; S <= P is the
// last level (one block per window, its U' is S_w).  Suffix sums of V by
// warp shuffles (five rounds in a warp, three across the block's warp
// totals), then the block sum of U + Suf_{+1} the same way: about 18
// dependent additions and three barriers per block, then log2 P doublings
// for V'.  A block's time is this chain's latency (measured the same as a
// shared-memory Hillis-Steele scan and tree of equal depth), so the
// levels cost about one block latency per wave of blocks: 16-bucket
// segments for 2^19 buckets keep the first upper level to one wave.
template <class F, int P>
__global__ void __launch_bounds__(P) k_wlevel(const XYZZ<F>* __restrict__ u_in, const XYZZ<F>* __restrict__ v_in,
                                              uint32_t S, XYZZ<F>* __restrict__ u_out, XYZZ<F>* __restrict__ v_out) {
    constexpr int NWARP = P / 32;
    static_assert(NWARP >= 1 && NWARP <= 32 && (NWARP & (NWARP - 1)) == 0, "block of 32..1024 threads, power of 2");
    __shared__ XYZZ<F> warp_v[NWARP], warp_later[NWARP], warp_x[NWARP];
    __shared__ XYZZ<F> block_v;
    const uint32_t nblk = S > (uint32_t)P ? S / P : 1u;
    const uint32_t w = blockIdx.x / nblk, k = blockIdx.x % nblk;
    const uint32_t width = S < (uint32_t)P ? S : (uint32_t)P;
    const uint32_t t = threadIdx.x;
    const int lane = (int)(t & 31), warp = (int)(t >> 5);
    const size_t idx = (size_t)w * S + (size_t)k * P + t;
    const bool live = t < width;
    // inclusive suffix sums of V inside the warp
    XYZZ<F> sv = live ? v_in[idx] : XYZZ<F>::inf();
#pragma unroll 1
    for (int d = 1; d < 32; d <<= 1) {
        const XYZZ<F> o = shfl_down_xyzz(sv, d);
        if (lane + d < 32) sv = wadd<F>(sv, o);
    }
    if (lane == 0) warp_v[warp] = sv;
    __syncthreads();
    // suffix sums over the warp totals (warp 0): later warps' V for every warp
    if (warp == 0) {
        XYZZ<F> c = lane < NWARP ? warp_v[lane] : XYZZ<F>::inf();
#pragma unroll 1
        for (int d = 1; d < NWARP; d <<= 1) {
            const XYZZ<F> o = shfl_down_xyzz(c, d);
            if (lane + d < NWARP) c = wadd<F>(c, o);
        }
        const XYZZ<F> after = shfl_down_xyzz(c, 1);
        if (lane < NWARP) warp_later[lane] = lane + 1 < NWARP ? after : XYZZ<F>::inf();
        if (lane == 0) block_v = c;
    }
    __syncthreads();
    // Suf_{t+1} + U_t
    const XYZZ<F> nxt = shfl_down_xyzz(sv, 1);
    XYZZ<F> x = wadd<F>(lane < 31 ? nxt : XYZZ<F>::inf(), warp_later[warp]);
    if (live) x = wadd<F>(x, u_in[idx]);
    // block sum: butterfly in the warp, then the warp sums in warp 0
#pragma unroll 1
    for (int d = 16; d >= 1; d >>= 1) {
        const XYZZ<F> o = shfl_down_xyzz(x, d);
        if (lane < d) x = wadd<F>(x, o);
    }
    if (lane == 0) warp_x[warp] = x;
    __syncthreads();
    if (warp == 0) {
        XYZZ<F> y = lane < NWARP ? warp_x[lane] : XYZZ<F>::inf();
#pragma unroll 1
        for (int d = NWARP / 2; d >= 1; d >>= 1) {
            const XYZZ<F> o = shfl_down_xyzz(y, d);
            if (lane < d) y = wadd<F>(y, o);
        }
        if (lane == 0) {
            u_out[blockIdx.x] = y;
            if (nblk > 1) {
                XYZZ<F> vsum = block_v;
                for (int i = 0; i < __builtin_ctz((unsigned)P); ++i) vsum = wdbl<F>(vsum);  // V' = P sum V
                v_out[blockIdx.x] = vsum;
            }
        }
    }
}

// Window multiples of resident bases: table[i W + w] = 2^(c w) P_i (affine,
// Montgomery).  One thread per base, c doublings per window, normalised with
// one inversion per warp per window (warp_batch_inverse: every lane takes
// part, so lanes past n carry infinity).
template <class F>
__global__ void __launch_bounds__(128) k_precompute(const Affine<F>* __restrict__ bases, uint64_t n, int W, int c,
                                                    Affine<F>* __restrict__ table) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    XYZZ<F> acc = active ? XYZZ<F>::from_affine(bases[i]) : XYZZ<F>::inf();
    for (int w = 0; w < W; ++w) {
        const bool inf = acc.is_inf();
        const F d = warp_batch_inverse<F>(inf ? F::one() : F::mul(acc.zz, acc.zzz));
        if (active) {
            table[i * (uint64_t)W + w] =
                inf ? Affine<F>::inf()
                    : Affine<F>{F::mul(acc.x, F::mul(d, acc.zzz)), F::mul(acc.y, F::mul(d, acc.zz))};
        }
        if (w + 1 < W)
            for (int k = 0; k < c; ++k) acc = XYZZ<F>::dbl(acc);
    }
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
__global__ void k_gather(const Affine<F>* __restrict__ bases, uint64_t nbases, int W, const uint64_t* __restrict__ idx,
                         uint64_t k, Affine<F>* __restrict__ out, uint32_t* __restrict__ first_bad) {
    // W entries per index: a table of window multiples (W = 1: the bases)
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= k * (uint64_t)W) return;
    const uint64_t j = t / (uint64_t)W, w = t % (uint64_t)W;
    const uint64_t i = idx[j];
    if (i >= nbases) { atomicMin(first_bad, (uint32_t)j); return; }
    out[t] = bases[i * W + w];
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

// Device tail of one MSM per thread: Horner over the set's window sums, then
// affine normalisation (infinity stays all-zero bytes).
template <class F>
__global__ void __launch_bounds__(64) k_msm_finish(const XYZZ<F>* __restrict__ win, uint32_t count, int W, int c,
                                                   const uint32_t* __restrict__ out_idx, uint8_t* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const XYZZ<F>* w = win + (size_t)k * W;
    XYZZ<F> acc = w[W - 1];
    for (int j = W - 2; j >= 0; --j) {
        if (!acc.is_inf())
            for (int d = 0; d < c; ++d) acc = XYZZ<F>::dbl(acc);
        acc = XYZZ<F>::add(acc, w[j]);
    }
    uint8_t* o = out + (size_t)(out_idx ? out_idx[k] : k) * 2 * sizeof(F);
    if (acc.is_inf()) {
        const uint4 z = make_uint4(0, 0, 0, 0);
        for (size_t b = 0; b < 2 * sizeof(F); b += 16) *reinterpret_cast<uint4*>(o + b) = z;
        return;
    }
    const Affine<F> a = acc.to_affine();
    store_canonical(o, a.x);
    store_canonical(o + sizeof(F), a.y);
}

template <class F>
struct HostOf;
template <>
struct HostOf<Fq> { typedef dvh::Fq T; };
template <>
struct HostOf<Fq2> { typedef dvh::Fq2 T; };

}  // namespace

// Default window width by size class: the autotuner's choices on B200 over
// 2^8..2^22 points, G1 and G2 alike.  Widths whose ceil(255 / c) windows
// leave few spare bits (5, 8, 10, 15, 16) win, by up to a quarter against
// the cost model's choice (2^16 points: c = 15 in 0.96 ms against the model's
// 13 in 1.28 ms).  0 outside the measured classes.
static int measured_c(uint64_t n) {
    int k = 0;
    while (k < 63 && (1ull << k) < n) ++k;
    if (k >= 8 && k <= 9) return 5;
    if (k >= 10 && k <= 12) return 8;
    if (k >= 13 && k <= 15) return 10;
    if (k >= 16 && k <= 20) return 15;
    if (k >= 21 && k <= 22) return 16;
    return 0;
}

int msm_seg_log(uint64_t all_buckets, uint32_t buckets, int c, bool g1) {
    // Long windows (a precomputed table's single bucket set of 2^18 or more
    // G1 buckets) take 16-bucket segments: fewer upper-level entries for a
    // modest first level (measured 0.86 instead of 1.06 ms at 2^19 buckets);
    // shorter windows and G2, whose additions cost three times as much,
    // keep 8.
    int seg_want = (g1 && buckets >= (1u << 18)) ? DV_SEG_LOG + 1 : DV_SEG_LOG;
    // Few buckets in all (sparse updates over a precomputed table, small
    // MSMs): the reduction is a latency chain, so keep about 2^15 first-level
    // threads and shorten the segments (128 buckets: one bucket each).
    int room = 0;
    while ((all_buckets >> (room + 1)) >= (1u << 15)) ++room;
    // Many buckets in all (a batch of sets over one table, 2^21 buckets or
    // more): longer segments, up to 64 buckets, while at least 2^17
    // first-level threads remain (several waves of k_segments at two blocks
    // per SM).  Each halving of the segment count halves the first upper
    // level, whose warp-0 phases and doublings leave most lanes idle.
    int wide = 0;
    while (wide < 6 && (all_buckets >> (wide + 1)) >= (1u << 17)) ++wide;
    seg_want = std::min(std::max(seg_want, wide), room);
    return std::min(seg_want, c - 1);
}

MsmPlan msm_plan(uint64_t n, int force_c) {
    MsmPlan p;
    int best_c = 4;
    double best = 1e300;
    for (int c = 4; c <= 20; ++c) {
        const double W = (255 + c - 1) / c;
        const double cost = W * (10.0 * (double)n + 28.0 * (double)(1u << (c - 1)));
        if (cost < best) { best = cost; best_c = c; }
    }
    if (const int m = measured_c(n)) best_c = m;
    p.c = force_c ? force_c : best_c;
    p.windows = (255 + p.c - 1) / p.c;
    p.buckets = 1u << (p.c - 1);
    p.seg_log = std::min(DV_SEG_LOG, p.c - 1);
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
    k_gather<F><<<blocks_for(k, 256), 256, 0, st>>>(d_bases, nbases, 1, d_idx, k, d_out, d_first_bad);
    DV_LAUNCH();
}

template <class F>
void gather_table(const Affine<F>* d_table, uint64_t nbases, int W, const uint64_t* d_idx, uint64_t k,
                  Affine<F>* d_out, uint32_t* d_first_bad, cudaStream_t st) {
    if (!k) return;
    k_gather<F><<<blocks_for(k * (uint64_t)W, 256), 256, 0, st>>>(d_table, nbases, W, d_idx, k, d_out, d_first_bad);
    DV_LAUNCH();
}
template void gather_table<Fq>(const Affine<Fq>*, uint64_t, int, const uint64_t*, uint64_t, Affine<Fq>*, uint32_t*,
                               cudaStream_t);

template <class F>
MsmPlan msm_plan_batch(uint32_t count, uint32_t max_set, uint64_t total, int force_c, const MsmPrecomp<F>* pre) {
    MsmPlan plan = msm_plan(max_set, force_c);
    if (!force_c && !pre && count > 1) {
        // every set carries windows * 2^(c-1) buckets: minimise
        // windows * (10 total + 2 * 28 * count * 2^(c-1)) (the reduction
        // runs at about half the accumulation's efficiency)
        double best = 1e300;
        for (int c = 4; c <= 20; ++c) {
            const double W = (255 + c - 1) / c;
            const double cost = W * (10.0 * (double)total + 56.0 * (double)count * (double)(1u << (c - 1)));
            if (cost < best) { best = cost; plan.c = c; }
        }
        plan.windows = (255 + plan.c - 1) / plan.c;
        plan.buckets = 1u << (plan.c - 1);
        plan.seg_log = std::min(DV_SEG_LOG, plan.c - 1);
    }
    // Bound the bucket table of a batch: count * windows * buckets <= 2^26
    // (8 GB of G1 XYZZ buckets); smaller windows trade buckets for windows.
    while (plan.c > 4 && (uint64_t)count * plan.windows * plan.buckets > (1ull << 26)) {
        plan.c--;
        plan.windows = (255 + plan.c - 1) / plan.c;
        plan.buckets = 1u << (plan.c - 1);
        plan.seg_log = std::min(DV_SEG_LOG, plan.c - 1);
    }
    if (pre) {
        // precomputed window multiples: the table fixes c and the window count
        plan.c = pre->c;
        plan.windows = pre->windows;
        plan.buckets = 1u << (plan.c - 1);
        plan.seg_log = std::min(DV_SEG_LOG, plan.c - 1);
    }
    return plan;
}

template <class F>
void msm_enqueue(MsmWorkspace& ws, const Affine<F>* d_points, const uint32_t* d_scalars, const SetMap& map,
                 uint32_t n, const MsmPlan& plan, const MsmPrecomp<F>* pre, uint32_t* d_err, cudaStream_t st) {
    const uint32_t count = map.count;
    const int c = plan.c, W = plan.windows;
    const uint32_t B = plan.buckets;
    const uint32_t Wr = pre ? 1u : (uint32_t)W;  // bucket sets (reduction windows) per MSM
    if (pre && (uint64_t)n * plan.windows >= (1ull << 31)) throw InvalidArgument("precomputed MSM too large");
    if ((uint64_t)count * Wr * plan.buckets > (1ull << 31) || (uint64_t)n * plan.windows > 0xffffffffull)
        throw InvalidArgument("MSM batch too large for one launch sequence");
    const uint32_t NW = count * Wr;
    const uint32_t NB = NW * B;

    uint32_t* d_counts = ws.counts.as<uint32_t>(NB);
    uint32_t* d_offsets = ws.offsets.as<uint32_t>(NB + 1);
    uint32_t* d_cursor = ws.cursor.as<uint32_t>(NB);
    uint32_t* d_sorted = ws.sorted.as<uint32_t>((size_t)n * W);
    XYZZ<F>* d_buckets = ws.buckets.as<XYZZ<F>>(NB);
    DV_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)NB * sizeof(uint32_t), st));

    MsmTimeline& tl = ws.timeline;
    auto mark = [&](int k) {
        if (tl.enabled) DV_CUDA(cudaEventRecord(tl.ev[k], st));
    };
    mark(0);
    if (pre) k_hist<true><<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, map, c, W, d_counts, d_err);
    else k_hist<false><<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, map, c, W, d_counts, d_err);
    DV_LAUNCH();
    mark(1);
    {
        const uint32_t ntiles = (NB + SCAN_TILE - 1) / SCAN_TILE;
        uint32_t* d_tiles = ws.scan_tiles.as<uint32_t>(ntiles);
        k_scan_tiles<<<ntiles, 1024, 0, st>>>(d_counts, NB, d_tiles);
        DV_LAUNCH();
        k_scan_top<<<1, 1024, 0, st>>>(d_tiles, ntiles, d_offsets + NB);
        DV_LAUNCH();
        k_scan_apply<<<ntiles, 1024, 0, st>>>(d_counts, NB, d_tiles, d_offsets, d_cursor);
        DV_LAUNCH();
    }
    mark(2);
    if (pre) k_scatter<true><<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, map, c, W, d_cursor, d_sorted);
    else k_scatter<false><<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, map, c, W, d_cursor, d_sorted);
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

    const int seg_log = plan.seg_force > 0 ? std::min(plan.seg_force, c - 1)
                                           : msm_seg_log((uint64_t)NW * B, B, c, sizeof(F) == sizeof(Fq));
    const uint32_t S = B >> seg_log;
    XYZZ<F>* d_seg_u = ws.segs.as<XYZZ<F>>(4ull * NW * S);
    XYZZ<F>* d_seg_r = d_seg_u + (size_t)NW * S;
    XYZZ<F>* d_lvl_u = d_seg_r + (size_t)NW * S;  // ping-pong buffers of the upper levels
    XYZZ<F>* d_lvl_r = d_lvl_u + (size_t)NW * S;
    XYZZ<F>* d_win = ws.windows.as<XYZZ<F>>(NW);
    constexpr int P = sizeof(F) == sizeof(Fq) ? 256 : 128;

    if (tl.enabled) DV_CUDA(cudaEventRecord(tl.acc_ev[0], st));
    k_accum<F><<<grid, 128, 0, st>>>(pre ? pre->table : d_points, d_sorted, d_offsets, NB, d_buckets, d_pgid, d_ppt);
    DV_LAUNCH();
    if (tl.enabled) DV_CUDA(cudaEventRecord(tl.acc_ev[1], st));
    uint32_t* d_fix_count = ws.fix_count.as<uint32_t>(1);
    uint32_t* d_fix_list = ws.fix_list.as<uint32_t>(T / FIX_SHORT + 1);
    DV_CUDA(cudaMemsetAsync(d_fix_count, 0, sizeof(uint32_t), st));
    k_fixup<F><<<blocks_for(T, 128), 128, 0, st>>>(d_pgid, d_ppt, T, d_buckets, d_fix_list, d_fix_count);
    DV_LAUNCH();
    // long chains are rare: a small grid loops over the queue
    k_fixup_long<F, 128><<<std::min<uint32_t>(T / FIX_SHORT + 1, (uint32_t)sm_count()), 128, 0, st>>>(
        d_pgid, d_ppt, T, d_buckets, d_fix_list, d_fix_count);
    DV_LAUNCH();
    mark(4);
    k_segments<F><<<blocks_for((uint64_t)NW * S, 128), 128, 0, st>>>(d_buckets, d_offsets, B, NW, seg_log, d_seg_u,
                                                                     d_seg_r);
    DV_LAUNCH();
    // upper levels: (U, V) pairs
    XYZZ<F>* u = d_seg_u;
    XYZZ<F>* r = d_seg_r;
    XYZZ<F>* u2 = d_lvl_u;
    XYZZ<F>* r2 = d_lvl_r;
    uint32_t len = S;
    for (;;) {
        const uint32_t nblk = len > (uint32_t)P ? len / P : 1u;
        XYZZ<F>* u_dst = nblk == 1 ? d_win : u2;
        k_wlevel<F, P><<<NW * nblk, P, 0, st>>>(u, r, len, u_dst, r2);
        DV_LAUNCH();
        if (nblk == 1) break;
        len = nblk;
        std::swap(u, u2);
        std::swap(r, r2);
    }
    mark(5);
}

template <class F>
void msm_run(MsmWorkspace& ws, const Affine<F>* d_points, const uint32_t* d_scalars, const uint32_t* set_offsets,
             uint32_t count, int force_c, cudaStream_t st, uint8_t* host_out, MsmStats* stats,
             const MsmPrecomp<F>* pre) {
    typedef typename HostOf<F>::T HF;
    const size_t out_bytes = 2 * sizeof(F);
    const uint32_t n = set_offsets[count];
    uint32_t max_set = 0;
    for (uint32_t k = 0; k < count; ++k) max_set = std::max(max_set, set_offsets[k + 1] - set_offsets[k]);
    if (n == 0 || count == 0) {
        memset(host_out, 0, (size_t)count * out_bytes);
        return;
    }
    const MsmPlan plan = msm_plan_batch<F>(count, max_set, n, force_c, pre);
    const int c = plan.c, W = plan.windows;
    const uint32_t Wr = pre ? 1u : (uint32_t)W;
    const uint32_t NW = count * Wr;

    uint32_t* d_set = ws.set_off.as<uint32_t>(count + 1);
    uint32_t* d_err = ws.err.as<uint32_t>(1);
    uint32_t* h_err = ws.host_err.as<uint32_t>(1);
    DV_CUDA(cudaMemcpyAsync(d_set, set_offsets, (count + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemsetAsync(d_err, 0xff, sizeof(uint32_t), st));
    msm_enqueue<F>(ws, d_points, d_scalars, SetMap{d_set, nullptr, count, 0}, n, plan, pre, d_err, st);

    XYZZ<F>* h_win = ws.host_windows.as<XYZZ<F>>(NW);
    DV_CUDA(cudaMemcpyAsync(h_win, ws.windows.as<XYZZ<F>>(NW), (size_t)NW * sizeof(XYZZ<F>), cudaMemcpyDeviceToHost,
                            st));
    DV_CUDA(cudaMemcpyAsync(h_err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (*h_err != NO_INDEX)
        throw InvalidArgument("non-canonical scalar at index " + std::to_string(*h_err));
    static_assert(sizeof(XYZZ<F>) == sizeof(dvh::XYZZ<HF>), "host/device XYZZ layout");
    const auto* hw = reinterpret_cast<const dvh::XYZZ<HF>*>(h_win);
    for (uint32_t k = 0; k < count; ++k) horner(hw + (size_t)k * Wr, (int)Wr, c, host_out + (size_t)k * out_bytes);
    MsmTimeline& tl = ws.timeline;
    if (tl.enabled) {
        DV_CUDA(cudaEventRecord(tl.ev[6], st));
        DV_CUDA(cudaEventSynchronize(tl.ev[6]));
        auto span = [&](cudaEvent_t a, cudaEvent_t b) {
            float ms = 0;
            DV_CUDA(cudaEventElapsedTime(&ms, a, b));
            return (double)ms;
        };
        const double acc = span(tl.acc_ev[0], tl.acc_ev[1]);
        tl.ms[0] += span(tl.ev[0], tl.ev[1]);        // digit histogram
        tl.ms[1] += span(tl.ev[1], tl.ev[2]);        // offsets scan
        tl.ms[2] += span(tl.ev[2], tl.ev[3]);        // scatter
        tl.ms[3] += acc;                             // bucket accumulation
        tl.ms[4] += span(tl.ev[3], tl.ev[4]) - acc;  // split-bucket merges
        tl.ms[5] += span(tl.ev[4], tl.ev[5]);        // bucket reduction
        tl.ms[7] += span(tl.ev[5], tl.ev[6]);        // window D2H + host Horner
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

// ---------------------------------------------------------------- direct small sparse MSMs
constexpr int SD_BLOCK = 256;
struct SdJob {
    uint32_t request, first, items, pad;  // terms first .. first + items - 1 (term = entry W + window)
};

// XYZZ point read past L1: written by another block of this launch (made
// visible by its __threadfence before the counter increment below).
DV_INL XYZZ<Fq> load_cg(const XYZZ<Fq>* p) {
    XYZZ<Fq> r;
    const uint4* src = reinterpret_cast<const uint4*>(p);
    uint4* dst = reinterpret_cast<uint4*>(&r);
    for (int i = 0; i < (int)(sizeof(XYZZ<Fq>) / 16); ++i) dst[i] = __ldcg(src + i);
    return r;
}

// Tree sum of sm[0 .. live) into sm[0] (entries up to the next power of two
// hold infinity): only the levels the live entries need.
DV_INL void block_sum(XYZZ<Fq>* sm, uint32_t live) {
    uint32_t span = 1;
    while (span < live) span <<= 1;
    for (uint32_t stride = span >> 1; stride > 0; stride >>= 1) {
        if (threadIdx.x < (unsigned)stride)
            sm[threadIdx.x] = XYZZ<Fq>::add_paired(sm[threadIdx.x], sm[threadIdx.x + stride]);
        __syncthreads();
    }
}

// Sparse MSMs over a window table in one launch.  Each block takes up to
// SD_BLOCK (entry, window) terms of one request: a thread forms d T (the
// signed c-bit digit d of the entry's window, T the table's multiple
// 2^(c w) P) by double-and-add, the block sums its threads.  The last block
// of a request to finish (a per-request counter, reset by that block for the
// next call) sums the request's block partials and writes the XYZZ sum.
// The host normalises all requests with one batch inversion, as the
// reference does (icicle_msm.cu:417-421): one thread's inversion on the
// device takes longer than that copy and a host batch inversion.
__global__ void __launch_bounds__(SD_BLOCK) k_sparse_direct(const G1A* __restrict__ table, uint64_t nbases, int c,
                                                            int W, const uint64_t* __restrict__ idx,
                                                            const uint32_t* __restrict__ vals,
                                                            const SdJob* __restrict__ jobs,
                                                            const uint32_t* __restrict__ req_blocks,
                                                            XYZZ<Fq>* __restrict__ partial, uint32_t* __restrict__ done,
                                                            XYZZ<Fq>* __restrict__ out, uint32_t* __restrict__ err) {
    __shared__ XYZZ<Fq> sm[SD_BLOCK];
    __shared__ bool last;
    const SdJob job = jobs[blockIdx.x];
    XYZZ<Fq> p = XYZZ<Fq>::inf();
    if (threadIdx.x < job.items) {
        const uint32_t term = job.first + threadIdx.x;
        const uint32_t e = term / (uint32_t)W, w = term % (uint32_t)W;
        uint32_t s[8];
        load_scalar(vals, e, s);
        const uint64_t ix = idx[e];
        if (!Fr::is_canonical(s)) {
            if (w == 0) atomicMin(err, e);
        } else if (ix >= nbases) {
            if (w == 0) atomicMin(err + 1, e);
        } else {
            // signed digit of window w (the recoding of k_hist)
            const uint32_t B = 1u << (c - 1), full = 1u << c;
            uint32_t carry = 0, mag = 0;
            bool neg = false;
            for (uint32_t v = 0; v <= w; ++v) {
                const uint32_t d = window_raw(s, (int)v * c, c) + carry;
                neg = d > B;
                mag = neg ? full - d : d;
                carry = neg ? 1u : 0u;
            }
            const G1A t = table[ix * (uint64_t)W + w];
            if (mag && !t.is_inf()) {
                p = XYZZ<Fq>::from_affine(t);
                for (int b = 30 - __clz(mag); b >= 0; --b) {
                    p = XYZZ<Fq>::dbl_paired(p);
                    if ((mag >> b) & 1) p = XYZZ<Fq>::add_affine(p, t);
                }
                if (neg) p = p.neg();
            }
        }
    }
    sm[threadIdx.x] = p;
    __syncthreads();
    block_sum(sm, job.items);
    const uint32_t r = job.request, b0 = req_blocks[r], b1 = req_blocks[r + 1];
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = sm[0];
        __threadfence();
        last = atomicAdd(done + r, 1u) == b1 - b0 - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    p = XYZZ<Fq>::inf();
    for (uint32_t b = b0 + threadIdx.x; b < b1; b += SD_BLOCK) p = XYZZ<Fq>::add_paired(p, load_cg(partial + b));
    sm[threadIdx.x] = p;
    __syncthreads();
    block_sum(sm, (b1 - b0) < (uint32_t)SD_BLOCK ? b1 - b0 : (uint32_t)SD_BLOCK);
    if (threadIdx.x == 0) {
        done[r] = 0;
        out[r] = sm[0];
    }
}

void msm_sparse_direct(MsmWorkspace& ws, const MsmPrecomp<Fq>& pre, uint64_t nbases, const uint64_t* d_idx,
                       const uint32_t* d_vals, const uint32_t* offs, uint32_t count, uint8_t* host_out,
                       cudaStream_t st) {
    const uint32_t W = (uint32_t)pre.windows;
    std::vector<SdJob> jobs;
    std::vector<uint32_t> req_blocks(count + 1, 0);
    bool empty = false;
    for (uint32_t r = 0; r < count; ++r) {
        const uint32_t first = offs[r] * W, terms = (offs[r + 1] - offs[r]) * W;
        for (uint32_t t = 0; t < terms; t += SD_BLOCK)
            jobs.push_back(SdJob{r, first + t, std::min<uint32_t>(SD_BLOCK, terms - t), 0});
        req_blocks[r + 1] = (uint32_t)jobs.size();
        empty |= terms == 0;
    }
    if (jobs.empty()) {
        memset(host_out, 0, (size_t)count * 64);
        return;
    }
    // one upload: the block list, then the per-request block offsets
    const size_t jb = jobs.size() * sizeof(SdJob), rb = (count + 1) * sizeof(uint32_t);
    uint8_t* h_desc = ws.host_desc.as<uint8_t>(jb + rb);
    memcpy(h_desc, jobs.data(), jb);
    memcpy(h_desc + jb, req_blocks.data(), rb);
    uint8_t* d_desc = ws.sd_jobs.as<uint8_t>(jb + rb);
    XYZZ<Fq>* d_partial = ws.sd_partial.as<XYZZ<Fq>>(jobs.size());
    uint32_t* d_done = ws.sd_req.as<uint32_t>(count);
    constexpr size_t XB = sizeof(XYZZ<Fq>);
    uint8_t* d_out = ws.sd_out.as<uint8_t>((size_t)count * XB + 16);
    uint32_t* d_err = reinterpret_cast<uint32_t*>(d_out + (size_t)count * XB);
    DV_CUDA(cudaMemcpyAsync(d_desc, h_desc, jb + rb, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemsetAsync(d_done, 0, count * sizeof(uint32_t), st));
    if (empty) DV_CUDA(cudaMemsetAsync(d_out, 0, (size_t)count * XB, st));  // all-zero XYZZ: infinity
    DV_CUDA(cudaMemsetAsync(d_err, 0xff, 2 * sizeof(uint32_t), st));
    k_sparse_direct<<<(unsigned)jobs.size(), SD_BLOCK, 0, st>>>(
        pre.table, nbases, pre.c, (int)W, d_idx, d_vals, reinterpret_cast<const SdJob*>(d_desc),
        reinterpret_cast<const uint32_t*>(d_desc + jb), d_partial, d_done, reinterpret_cast<XYZZ<Fq>*>(d_out), d_err);
    DV_LAUNCH();
    // one copy back: the results, then the two error words
    uint8_t* h_out = ws.host_windows.as<uint8_t>((size_t)count * XB + 16);
    DV_CUDA(cudaMemcpyAsync(h_out, d_out, (size_t)count * XB + 8, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    uint32_t h_err[2];
    memcpy(h_err, h_out + (size_t)count * XB, 8);
    if (h_err[0] != NO_INDEX) throw InvalidArgument("non-canonical scalar at index " + std::to_string(h_err[0]));
    if (h_err[1] != NO_INDEX) throw InvalidArgument("sparse MSM index out of range");
    static_assert(sizeof(XYZZ<Fq>) == sizeof(dvh::XYZZ<dvh::Fq>), "host/device XYZZ layout");
    dvh::xyzz_batch_to_affine_bytes(reinterpret_cast<const dvh::XYZZ<dvh::Fq>*>(h_out), count, host_out);
}

template void msm_run<Fq>(MsmWorkspace&, const Affine<Fq>*, const uint32_t*, const uint32_t*, uint32_t, int,
                          cudaStream_t, uint8_t*, MsmStats*, const MsmPrecomp<Fq>*);
template void msm_run<Fq2>(MsmWorkspace&, const Affine<Fq2>*, const uint32_t*, const uint32_t*, uint32_t, int,
                           cudaStream_t, uint8_t*, MsmStats*, const MsmPrecomp<Fq2>*);
template MsmPlan msm_plan_batch<Fq>(uint32_t, uint32_t, uint64_t, int, const MsmPrecomp<Fq>*);
template MsmPlan msm_plan_batch<Fq2>(uint32_t, uint32_t, uint64_t, int, const MsmPrecomp<Fq2>*);
template void msm_enqueue<Fq>(MsmWorkspace&, const Affine<Fq>*, const uint32_t*, const SetMap&, uint32_t,
                              const MsmPlan&, const MsmPrecomp<Fq>*, uint32_t*, cudaStream_t);
template void msm_enqueue<Fq2>(MsmWorkspace&, const Affine<Fq2>*, const uint32_t*, const SetMap&, uint32_t,
                               const MsmPlan&, const MsmPrecomp<Fq2>*, uint32_t*, cudaStream_t);

template <class F>
void msm_finish_device(const XYZZ<F>* d_windows, uint32_t count, int windows_per_set, int c, const uint32_t* d_out_idx,
                       uint8_t* d_out, cudaStream_t st) {
    if (!count) return;
    k_msm_finish<F><<<blocks_for(count, 64), 64, 0, st>>>(d_windows, count, windows_per_set, c, d_out_idx, d_out);
    DV_LAUNCH();
}
template void msm_finish_device<Fq>(const XYZZ<Fq>*, uint32_t, int, int, const uint32_t*, uint8_t*, cudaStream_t);
template void msm_finish_device<Fq2>(const XYZZ<Fq2>*, uint32_t, int, int, const uint32_t*, uint8_t*, cudaStream_t);

template <class F>
void msm_precompute(const Affine<F>* d_bases, uint64_t n, int c, int windows, Affine<F>* d_table, cudaStream_t st) {
    if (!n) return;
    k_precompute<F><<<blocks_for(n, 128), 128, 0, st>>>(d_bases, n, windows, c, d_table);
    DV_LAUNCH();
}
template void msm_precompute<Fq>(const Affine<Fq>*, uint64_t, int, int, Affine<Fq>*, cudaStream_t);
template void msm_precompute<Fq2>(const Affine<Fq2>*, uint64_t, int, int, Affine<Fq2>*, cudaStream_t);

MsmPlan msm_plan_precomputed(uint64_t n) {
    // one shared bucket set: windows * 10 n additions + 28 * 2^(c-1) for the reduction
    MsmPlan p{};
    double best = 1e300;
    for (int c = 8; c <= 22; ++c) {
        const double W = (255 + c - 1) / c;
        const double cost = W * 10.0 * (double)n + 28.0 * (double)(1u << (c - 1));
        if (cost < best) { best = cost; p.c = c; }
    }
    p.windows = (255 + p.c - 1) / p.c;
    p.buckets = 1u << (p.c - 1);
    p.seg_log = std::min(DV_SEG_LOG, p.c - 1);
    return p;
}
template void convert_points<Fq>(const uint8_t*, Affine<Fq>*, uint64_t, uint32_t*, cudaStream_t);
template void convert_points<Fq2>(const uint8_t*, Affine<Fq2>*, uint64_t, uint32_t*, cudaStream_t);
template void gather_points<Fq>(const Affine<Fq>*, uint64_t, const uint64_t*, uint64_t, Affine<Fq>*, uint32_t*,
                                cudaStream_t);
template void gather_points<Fq2>(const Affine<Fq2>*, uint64_t, const uint64_t*, uint64_t, Affine<Fq2>*, uint32_t*,
                                 cudaStream_t);

}  // namespace dv
