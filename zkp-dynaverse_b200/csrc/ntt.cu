// Fr NTT kernels and launch sequence (see ntt.cuh).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>

#include "curve.cuh"
#include "ntt.cuh"

namespace dv {

namespace {

// TWO_ADIC_ROOT_OF_UNITY of BN254 Fr: 5^((r-1)/2^28), canonical limbs.
__device__ __constant__ uint32_t ROOT28[8] = {0x725b19f0u, 0x9bd61b6eu, 0x41112ed4u, 0x402d111eu,
                                              0x8ef62abcu, 0x00e0a7ebu, 0xa58a7e85u, 0x2a3c09f0u};

// consts layout (Fr, Montgomery unless noted):
//  0: w (order n; inverted for inverse kinds)   1: n^-1   2: n^-1 (canonical)
//  3: g = 5   4: g^-1   5: g^(2^split)   6: g^-(2^split)   7: R (= R2 as Montgomery)
//  8: one (canonical 1)
enum { C_W = 0, C_NINV, C_NINV_CANON, C_G, C_GINV, C_G_SPLIT, C_GINV_SPLIT, C_R, C_ONE_RAW, C_COUNT };

__global__ void k_setup_consts(int logn, int inverse, int split, Fr* out) {
    if (threadIdx.x || blockIdx.x) return;
    uint32_t rc[8];
    for (int i = 0; i < 8; ++i) rc[i] = ROOT28[i];
    Fr w = Fr::from_canonical(rc);
    for (int k = logn; k < 28; ++k) w = Fr::sqr(w);
    if (inverse) w = Fr::inv(w);
    uint32_t nc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    nc[logn / 32] = 1u << (logn % 32);
    const Fr nm = Fr::from_canonical(nc);
    const Fr ninv = Fr::inv(nm);
    uint32_t gc[8] = {5, 0, 0, 0, 0, 0, 0, 0};
    const Fr g = Fr::from_canonical(gc);
    const Fr ginv = Fr::inv(g);
    Fr gs = g, gis = ginv;
    for (int k = 0; k < split; ++k) { gs = Fr::sqr(gs); gis = Fr::sqr(gis); }
    const Fr r2 = Fr::r2();
    uint32_t canon[8];
    ninv.to_canonical(canon);
    Fr ninv_c;
    for (int i = 0; i < 8; ++i) ninv_c.v[i] = canon[i];
    Fr one_raw = Fr::zero();
    one_raw.v[0] = 1;
    out[C_W] = w;
    out[C_NINV] = ninv;
    out[C_NINV_CANON] = ninv_c;
    out[C_G] = g;
    out[C_GINV] = ginv;
    out[C_G_SPLIT] = gs;
    out[C_GINV_SPLIT] = gis;
    out[C_R] = r2;
    out[C_ONE_RAW] = one_raw;
}

// out[i] = base^i * mul for i < count (Montgomery), computed in chunks of
// `chunk` consecutive powers per thread.  canonical_out converts to canonical.
__global__ void k_pow_table(const Fr* __restrict__ base_p, const Fr* __restrict__ mul_p, uint64_t count,
                            uint32_t chunk, int canonical_out, Fr* __restrict__ out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t start = t * chunk;
    if (start >= count) return;
    const Fr base = *base_p;
    // x = base^start
    Fr x = Fr::one();
    for (int bit = 63 - __clzll(start | 1); bit >= 0; --bit) {
        x = Fr::sqr(x);
        if ((start >> bit) & 1) x = Fr::mul(x, base);
    }
    const uint64_t end = min(count, start + chunk);
    for (uint64_t i = start; i < end; ++i) {
        Fr v = mul_p ? Fr::mul(x, *mul_p) : x;
        if (canonical_out) {
            uint32_t c[8];
            v.to_canonical(c);
            for (int j = 0; j < 8; ++j) v.v[j] = c[j];
        }
        out[i] = v;
        x = Fr::mul(x, base);
    }
}

// Shared-memory staging: two planes of 16-byte halves (plane 0: words 0-3 of
// every element, plane 1: words 4-7), so an element moves with two 128-bit
// accesses.  A 128-bit access is served eight threads at a time, one
// 128-byte row of 8 slots, so eight threads must hit eight distinct slots
// (index mod 8).  Within a round, the eight threads' element indices differ
// in three bits taken from {0..5} (the low tau bits land on element bits
// [0, b_lo) and [b_lo + RR, ...)).  The slot is e XOR S(e[3..5]) with
// S linear over GF(2): e3 -> 7, e4 -> 5, e5 -> 6; for every (b_lo, RR) with
// RR <= 3 the three varying bits map to independent slot vectors, so the
// rows are conflict-free.  SWZ packs S(b) for b = 0..7 in nibbles.
constexpr uint32_t SWZ = 0x43162570u;
DV_INL uint32_t slot(uint32_t e) { return e ^ ((SWZ >> (((e >> 3) & 7u) << 2)) & 7u); }
DV_INL void load_plane(const uint32_t* sm, uint32_t n, uint32_t e, Fr& a) {
    const uint4* s4 = reinterpret_cast<const uint4*>(sm);
    const uint32_t o = slot(e);
    const uint4 lo = s4[o], hi = s4[n + o];
    a.v[0] = lo.x; a.v[1] = lo.y; a.v[2] = lo.z; a.v[3] = lo.w;
    a.v[4] = hi.x; a.v[5] = hi.y; a.v[6] = hi.z; a.v[7] = hi.w;
}
DV_INL void store_plane(uint32_t* sm, uint32_t n, uint32_t e, const Fr& a) {
    uint4* s4 = reinterpret_cast<uint4*>(sm);
    const uint32_t o = slot(e);
    s4[o] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
    s4[n + o] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

// Arguments of one DIF pass (kernel parameters, passed by value).
struct PassArgs {
    const uint8_t* in;        // first pass: canonical input bytes
    Fr* work;                 // working vector (bit-reversed order after the last pass)
    uint8_t* out;             // non-null on a fused last pass: natural-order output bytes
    const Fr* tw;             // w^i, i < n/2
    const Fr* pre_hi;         // coset pre-scale g^i (two-level table), first pass only
    const Fr* pre_lo;
    const Fr* post_hi;        // fused last pass: coset post-scale g^-i n^-1
    const Fr* post_lo;
    const Fr* post_const;     // fused last pass: n^-1 (plain inverse)
    uint32_t* first_bad;      // lowest non-canonical input index
    int logn, s0, k, first, split;
};

// One DIF pass over stages [s0, s0 + k) for one group of G = 2^k elements
// (stride 2^lb in the vector).  Register-blocked: the k stages are processed
// in rounds of up to R = 2^R_LOG elements per thread; a round loads R
// elements that differ only in its bits, runs its radix-2 stages in
// registers and writes them back, so shared memory is touched once per
// round rather than once per stage.  The first round reads global memory
// directly (first pass: canonical check and coset pre-scale); the last round
// writes global memory directly: the working vector, or, on a fused last
// pass, the output bytes at the bit-reversed position with the inverse or
// coset post-scale applied.
// One round of RR stages: thread-group tau owns the 2^RR elements that differ
// only in local bits [bit_hi - RR, bit_hi).  RR is a compile-time constant so
// the element array stays in registers.
// Working-vector load that bypasses L1: in a batch, a later pass reads
// elements that other blocks of the same launch wrote.
DV_INL Fr load_cg(const Fr* p) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    const uint4 lo = __ldcg(q), hi = __ldcg(q + 1);
    Fr a;
    a.v[0] = lo.x; a.v[1] = lo.y; a.v[2] = lo.z; a.v[3] = lo.w;
    a.v[4] = hi.x; a.v[5] = hi.y; a.v[6] = hi.z; a.v[7] = hi.w;
    return a;
}

// The tile holds 2^tile_log elements: groups first_group, first_group + 1, ...
// of 2^k elements each.  Tile index t = (group in tile) << k | element in
// group, so the round's lane -> element formula covers every group at once.
template <int RR, int THREADS, bool CG>
DV_INL void dif_round(const PassArgs& a, uint32_t* sm, int tile_log, uint64_t first_group, int bit_hi,
                      bool first_round) {
    constexpr int R = 1 << RR;
    const int k = a.k;
    const int lb = a.logn - a.s0 - k;
    const uint32_t G = 1u << k;
    const uint32_t TE = 1u << tile_log;
    const int b_lo = bit_hi - RR;
    const bool last_round = b_lo == 0;
    const uint32_t lanes = TE >> RR;
    for (uint32_t tau = threadIdx.x; tau < lanes; tau += THREADS) {
        const uint32_t base_t = ((tau >> b_lo) << bit_hi) | (tau & ((1u << b_lo) - 1));
        const uint64_t g = first_group + (base_t >> k);
        const uint64_t low = g & ((1ull << lb) - 1), high = g >> lb;
        const uint32_t base_e = base_t & (G - 1);
        Fr x[R];
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const uint32_t e = base_e | ((uint32_t)m << b_lo);
            const uint64_t idx = (high << (lb + k)) | ((uint64_t)e << lb) | low;
            if (first_round) {
                if (a.first) {
                    uint32_t c[8];
                    load_words(a.in + 32 * idx, c);
                    if (!Fr::is_canonical(c)) {
                        atomicMin(a.first_bad, (uint32_t)idx);
#pragma unroll
                        for (int j = 0; j < 8; ++j) c[j] = 0;
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j) x[m].v[j] = c[j];
                    // values stay canonical: multipliers are held in
                    // Montgomery form and mont_mul(a, x R) = a x
                    if (a.pre_hi) {
                        const uint64_t lo_mask = (1ull << a.split) - 1;
                        x[m] = Fr::mul_inl(Fr::mul_inl(x[m], a.pre_hi[idx >> a.split]), a.pre_lo[idx & lo_mask]);
                    }
                } else {
                    x[m] = CG ? load_cg(a.work + idx) : a.work[idx];
                }
            } else {
                load_plane(sm, TE, base_t | ((uint32_t)m << b_lo), x[m]);
            }
        }
#pragma unroll
        for (int j = 0; j < RR; ++j) {
            const int s = a.s0 + (k - bit_hi) + j;  // global stage
            const int pb = bit_hi - 1 - j;          // local bit of this stage
            const int hs = 1 << (RR - 1 - j);      // pair distance in m
            // issue this stage's twiddle loads before its butterflies
            Fr w[R / 2];
#pragma unroll
            for (int m = 0, q = 0; m < R; ++m) {
                if (m & hs) continue;
                const uint32_t e = base_e | ((uint32_t)m << b_lo);
                const uint64_t jp = ((uint64_t)(e & ((1u << pb) - 1)) << lb) | low;
                w[q++] = a.tw[jp << s];
            }
#pragma unroll
            for (int m = 0, q = 0; m < R; ++m) {
                if (m & hs) continue;
                const Fr u = x[m], v = x[m + hs];
                x[m] = Fr::add(u, v);
                x[m + hs] = Fr::mul_inl(Fr::sub(u, v), w[q++]);
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const uint32_t e = base_e | ((uint32_t)m << b_lo);
            if (last_round) {
                const uint64_t idx = (high << (lb + k)) | ((uint64_t)e << lb) | low;
                if (a.out) {
                    const uint64_t i = __brevll(idx) >> (64 - a.logn);
                    Fr y = x[m];
                    if (a.post_hi) {
                        const uint64_t lo_mask = (1ull << a.split) - 1;
                        y = Fr::mul_inl(Fr::mul_inl(y, a.post_hi[i >> a.split]), a.post_lo[i & lo_mask]);
                    } else if (a.post_const) {
                        y = Fr::mul_inl(y, *a.post_const);
                    }
                    store_words(a.out + 32 * i, y.v);
                } else {
                    a.work[idx] = x[m];
                }
            } else {
                store_plane(sm, TE, base_t | ((uint32_t)m << b_lo), x[m]);
            }
        }
    }
}

// Runs the rounds of one tile (all stages of the pass), ending with a
// barrier.
template <int THREADS, int R_LOG, bool CG>
DV_INL void dif_tile(const PassArgs& a, uint32_t* sm, int tile_log, uint64_t first_group) {
    int bit_hi = a.k;
    bool first_round = true;
    while (bit_hi > 0) {
        const int rr = bit_hi < R_LOG ? bit_hi : R_LOG;
        if (rr == 3 && R_LOG >= 3)
            dif_round<(R_LOG >= 3 ? 3 : 1), THREADS, CG>(a, sm, tile_log, first_group, bit_hi, first_round);
        else if (rr == 2) dif_round<2, THREADS, CG>(a, sm, tile_log, first_group, bit_hi, first_round);
        else dif_round<1, THREADS, CG>(a, sm, tile_log, first_group, bit_hi, first_round);
        __syncthreads();
        bit_hi -= rr;
        first_round = false;
    }
}

#ifndef DV_NTT_MINB
#define DV_NTT_MINB 3
#endif
#ifndef DV_NTT_RADIX_LOG
#define DV_NTT_RADIX_LOG 2
#endif
template <int THREADS, int R_LOG>
__global__ void __launch_bounds__(THREADS, (THREADS >= 256 ? DV_NTT_MINB : 8)) k_dif_pass(const PassArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    const int k = a.k;
    const int lb = a.logn - a.s0 - k;
    const uint64_t g = blockIdx.x;
    const uint64_t low = g & ((1ull << lb) - 1), high = g >> lb;
    dif_tile<THREADS, R_LOG, false>(a, sm, k, g);
    if (k == 0) {  // single element: copy (with the first pass's check)
        if (threadIdx.x == 0) {
            const uint64_t idx = (high << lb) | low;
            Fr v;
            if (a.first) {
                uint32_t c[8];
                load_words(a.in + 32 * idx, c);
                if (!Fr::is_canonical(c)) {
                    atomicMin(a.first_bad, (uint32_t)idx);
                    for (int j = 0; j < 8; ++j) c[j] = 0;
                }
                for (int j = 0; j < 8; ++j) v.v[j] = c[j];
                if (a.pre_hi) v = Fr::mul_inl(Fr::mul_inl(v, a.pre_hi[0]), a.pre_lo[0]);
            } else {
                v = a.work[idx];
            }
            a.work[idx] = v;
        }
    }
}

// Bit-reversal permutation + post scaling (values are already canonical).
__global__ void k_permute(const Fr* __restrict__ work, uint8_t* __restrict__ out, int logn,
                          const Fr* __restrict__ post_hi, const Fr* __restrict__ post_lo, int split,
                          const Fr* __restrict__ post_const) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >> logn) return;
    const uint64_t r = logn ? (__brevll(i) >> (64 - logn)) : 0;
    Fr a = work[r];
    if (post_hi) {
        const uint64_t lo_mask = (1ull << split) - 1;
        a = Fr::mul_inl(Fr::mul_inl(a, post_hi[i >> split]), post_lo[i & lo_mask]);
    } else if (post_const) {
        a = Fr::mul_inl(a, *post_const);
    }
    store_words(out + 32 * i, a.v);
}

constexpr int MAX_DEVICES = 64;

template <int THREADS>
void launch_pass(const PassArgs& a, cudaStream_t st) {
    const size_t smem = (size_t)32 << a.k;  // two planes of 16 bytes per element
    static std::atomic<bool> configured[MAX_DEVICES] = {};
    int dev = 0;
    DV_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) throw InvalidArgument("device ordinal out of range");
    if (!configured[dev].load(std::memory_order_acquire)) {
        // idempotent: threads racing here set the same attribute
        DV_CUDA(cudaFuncSetAttribute(k_dif_pass<THREADS, DV_NTT_RADIX_LOG>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
        configured[dev].store(true, std::memory_order_release);
    }
    const unsigned groups = 1u << (a.logn - a.k);
    k_dif_pass<THREADS, DV_NTT_RADIX_LOG><<<groups, THREADS, smem, st>>>(a);
    DV_LAUNCH();
}

// Runs the DIF passes of a transform of 2^logn elements.  With fuse_out the
// last pass writes the natural-order output bytes itself.  In-place use is
// safe: the first pass reads the input and a later pass writes the output;
// a single pass is one block whose first round reads every element before
// a barrier (or, with one round, one thread reading all before writing) and
// whose last round writes.  Returns whether the output was written
// (otherwise k_permute must run).
bool run_passes(const uint8_t* d_in, Fr* work, uint8_t* d_out, int logn, const Fr* tw, const Fr* pre_hi,
                const Fr* pre_lo, const Fr* post_hi, const Fr* post_lo, const Fr* post_const, int split,
                uint32_t* bad, bool fuse_out, cudaStream_t st) {
    PassArgs a{d_in, work, nullptr, tw, pre_hi, pre_lo, post_hi, post_lo, post_const, bad, logn, 0, 0, 1, split};
    if (logn == 0) {
        // single element: conversion round trip checks canonical form
        launch_pass<32>(a, st);
        return false;
    }
    const int passes = (logn + 10) / 11;
    const bool fused = fuse_out;
    int s0 = 0;
    for (int p = 0; p < passes; ++p) {
        a.k = logn / passes + (p < logn % passes ? 1 : 0);
        a.s0 = s0;
        a.first = p == 0;
        a.out = (fused && p == passes - 1) ? d_out : nullptr;
        if (a.k >= 9) launch_pass<256>(a, st);
        else launch_pass<64>(a, st);
        s0 += a.k;
    }
    return fused;
}

}  // namespace

NttTables& ntt_tables(NttWorkspace& ws, int logn, int kind, cudaStream_t st) {
    if (logn < 0 || logn > NTT_MAX_LOG || kind < 0 || kind > 3) throw InvalidArgument("invalid NTT size or kind");
    const uint64_t n = 1ull << logn;
    const bool inverse = kind & 1, coset = kind >= 2;
    const int split = (logn + 1) / 2;
    const int key = logn * 4 + kind;
    auto it = ws.tables.find(key);
    if (it != ws.tables.end()) return *it->second;
    auto t = std::make_unique<NttTables>();
    t->split = split;
    Fr* kc = t->consts.as<Fr>(C_COUNT);
    k_setup_consts<<<1, 1, 0, st>>>(logn, inverse ? 1 : 0, split, kc);
    DV_LAUNCH();
    const uint64_t half = std::max<uint64_t>(1, n / 2);
    Fr* tw = t->tw.as<Fr>(half);
    const uint32_t chunk = 64;
    const uint64_t threads = (half + chunk - 1) / chunk;
    k_pow_table<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(kc + C_W, nullptr, half, chunk, 0, tw);
    DV_LAUNCH();
    if (coset) {
        const uint64_t nlo = 1ull << split, nhi = (n + nlo - 1) >> split;
        if (!inverse) {
            Fr* hi = t->pre_hi.as<Fr>(nhi);
            Fr* lo = t->pre_lo.as<Fr>(nlo);
            k_pow_table<<<(unsigned)((nhi + 127) / 128), 128, 0, st>>>(kc + C_G_SPLIT, nullptr, nhi, 1, 0, hi);
            DV_LAUNCH();
            k_pow_table<<<(unsigned)((nlo + 127) / 128), 128, 0, st>>>(kc + C_G, nullptr, nlo, 1, 0, lo);
            DV_LAUNCH();
        } else {
            Fr* hi = t->post_hi.as<Fr>(nhi);
            Fr* lo = t->post_lo.as<Fr>(nlo);
            k_pow_table<<<(unsigned)((nhi + 127) / 128), 128, 0, st>>>(kc + C_GINV_SPLIT, kc + C_NINV, nhi, 1, 0, hi);
            DV_LAUNCH();
            k_pow_table<<<(unsigned)((nlo + 127) / 128), 128, 0, st>>>(kc + C_GINV, nullptr, nlo, 1, 0, lo);
            DV_LAUNCH();
        }
    }
    NttTables& ref = *t;
    ws.tables[key] = std::move(t);
    return ref;
}

const uint32_t* ntt_ninv_canonical(NttTables& tables) {
    return reinterpret_cast<const uint32_t*>(tables.consts.as<Fr>(C_COUNT) + C_NINV_CANON);
}

namespace {
// Multipliers of one transform, taken from its tables.
struct Scaling {
    const Fr *tw, *pre_hi, *pre_lo, *post_hi, *post_lo, *post_const;
    int split;
};
Scaling scaling_of(NttTables& tab, int kind) {
    const bool inverse = kind & 1, coset = kind >= 2;
    Fr* kc = tab.consts.as<Fr>(C_COUNT);
    return Scaling{tab.tw.as<Fr>(1),
                   (coset && !inverse) ? tab.pre_hi.as<Fr>(1) : nullptr,
                   (coset && !inverse) ? tab.pre_lo.as<Fr>(1) : nullptr,
                   (coset && inverse) ? tab.post_hi.as<Fr>(1) : nullptr,
                   (coset && inverse) ? tab.post_lo.as<Fr>(1) : nullptr,
                   inverse ? kc + C_NINV : nullptr,
                   tab.split};
}
}  // namespace

void ntt_run(NttWorkspace& ws, const uint8_t* d_in, uint8_t* d_out, int logn, int kind, cudaStream_t st) {
    NttTables& tab = ntt_tables(ws, logn, kind, st);
    const uint64_t n = 1ull << logn;
    const Scaling sc = scaling_of(tab, kind);
    Fr* work = ws.work.as<Fr>(n);
    uint32_t* bad = ws.err.as<uint32_t>(1);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), st));

    if (!run_passes(d_in, work, d_out, logn, sc.tw, sc.pre_hi, sc.pre_lo, sc.post_hi, sc.post_lo, sc.post_const,
                    sc.split, bad, true, st)) {
        k_permute<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(work, d_out, logn, sc.post_hi, sc.post_lo, sc.split,
                                                              sc.post_const);
        DV_LAUNCH();
    }
    uint32_t host_bad = 0;
    DV_CUDA(cudaMemcpyAsync(&host_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (host_bad != 0xffffffffu) throw InvalidArgument("non-canonical NTT input at index " + std::to_string(host_bad));
    ws.calls++;
    ws.elements += n;
}

// ===================================================================== batches
namespace {

constexpr uint32_t BATCH_SPIN_LIMIT = 1u << 24;  // dependency wait: ~2 s of 128 ns sleeps

struct BatchDesc {
    PassArgs a;         // k, s0, first and out are set per pass
    int passes;
    int k[3], s0[3], tile_log[3];
    uint32_t tiles[3];  // tiles of each pass
};
struct BatchTile {
    uint32_t desc;
    uint32_t pass;
    uint64_t first_group;
};

// Persistent batch kernel.  ctl[0]: next tile, ctl[1]: status (bit 0: a
// dependency wait gave up), ctl[2 + 3 d + p]: finished tiles of pass p of
// transform d.  Tiles are listed pass by pass, so a tile only waits for
// tiles that running blocks took earlier.
// Radix 8 holds 8 elements and 4 twiddles in registers: it gets two
// resident blocks (128 registers) instead of three.
template <int R_LOG>
__global__ void __launch_bounds__(256, R_LOG >= 3 ? 2 : DV_NTT_MINB) k_ntt_batch(const BatchDesc* __restrict__ descs,
                                                                const BatchTile* __restrict__ tiles, uint32_t ntiles,
                                                                uint32_t* __restrict__ ctl) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint32_t cur;
    for (;;) {
        if (threadIdx.x == 0) cur = atomicAdd(ctl, 1u);
        __syncthreads();
        const uint32_t t = cur;
        if (t >= ntiles) return;
        const BatchTile tile = tiles[t];
        const BatchDesc& d = descs[tile.desc];
        const int p = (int)tile.pass;
        if (p > 0) {
            if (threadIdx.x == 0) {
                const volatile uint32_t* dep = ctl + 2 + 3 * tile.desc + (p - 1);
                const uint32_t need = d.tiles[p - 1];
                uint32_t spins = 0;
                while (*dep < need) {
                    if (++spins > BATCH_SPIN_LIMIT) {
                        atomicOr(ctl + 1, 1u);
                        break;
                    }
                    __nanosleep(128);
                }
                __threadfence();
            }
            __syncthreads();
        }
        PassArgs a = d.a;
        a.k = d.k[p];
        a.s0 = d.s0[p];
        a.first = p == 0;
        a.out = p == d.passes - 1 ? d.a.out : nullptr;
        dif_tile<256, R_LOG, true>(a, sm, d.tile_log[p], tile.first_group);  // ends with a barrier
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(ctl + 2 + 3 * tile.desc + p, 1u);
        }
    }
}

}  // namespace

void ntt_batch_prepare(NttWorkspace& ws, NttBatch& batch, const std::vector<NttBatchItem>& items, cudaStream_t st,
                       int tile_log) {
    if (tile_log < BATCH_TILE_MIN || tile_log > BATCH_TILE_MAX) throw InvalidArgument("batch NTT tile out of range");
    const uint32_t count = (uint32_t)items.size();
    std::vector<BatchDesc> descs(count);
    std::vector<BatchTile> tiles[3];
    batch.work_off.assign(count, 0);
    uint64_t total = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const NttBatchItem& it = items[i];
        if (it.logn < 1 || it.logn > 24 || it.kind < 0 || it.kind > 3 || !it.in || !it.out)
            throw InvalidArgument("invalid batch NTT item " + std::to_string(i));
        batch.work_off[i] = total;
        total += 1ull << it.logn;
    }
    if (total > (1ull << 30)) throw InvalidArgument("NTT batch too large");
    Fr* work = batch.work.as<Fr>(std::max<uint64_t>(1, total));
    uint32_t* errs = batch.errs.as<uint32_t>(std::max<uint32_t>(1, count));
    for (uint32_t i = 0; i < count; ++i) {
        const NttBatchItem& it = items[i];
        const Scaling sc = scaling_of(ntt_tables(ws, it.logn, it.kind, st), it.kind);
        BatchDesc& d = descs[i];
        d.a = PassArgs{it.in,       work + batch.work_off[i], it.out, sc.tw,    sc.pre_hi, sc.pre_lo,
                       sc.post_hi, sc.post_lo,               sc.post_const,    errs + i, it.logn,  0,
                       0,          1,                        sc.split};
        d.passes = (it.logn + tile_log - 1) / tile_log;  // at most 3: logn <= 24, tile_log >= 8
        for (int p = 0; p < 3; ++p) {
            d.k[p] = d.s0[p] = d.tile_log[p] = 0;
            d.tiles[p] = 0;
        }
        int s0 = 0;
        for (int p = 0; p < d.passes; ++p) {
            const int k = it.logn / d.passes + (p < it.logn % d.passes ? 1 : 0);
            const int tl = std::min(it.logn, tile_log);  // 2^(tl - k) groups of 2^k per tile
            const uint64_t groups = 1ull << (it.logn - k);
            const uint64_t per_tile = 1ull << (tl - k);
            d.k[p] = k;
            d.s0[p] = s0;
            d.tile_log[p] = tl;
            d.tiles[p] = (uint32_t)(groups / per_tile);
            for (uint64_t g = 0; g < groups; g += per_tile) tiles[p].push_back(BatchTile{i, (uint32_t)p, g});
            s0 += k;
        }
    }
    std::vector<BatchTile> all;
    for (auto& v : tiles) all.insert(all.end(), v.begin(), v.end());
    batch.count = count;
    batch.ntiles = (uint32_t)all.size();
    batch.elements = total;
    BatchDesc* d_descs = batch.descs.as<BatchDesc>(std::max<uint32_t>(1, count));
    BatchTile* d_tiles = batch.tiles.as<BatchTile>(std::max<size_t>(1, all.size()));
    batch.ctl.as<uint32_t>(2 + 3ull * count);
    if (count) DV_CUDA(cudaMemcpyAsync(d_descs, descs.data(), count * sizeof(BatchDesc), cudaMemcpyHostToDevice, st));
    if (!all.empty())
        DV_CUDA(cudaMemcpyAsync(d_tiles, all.data(), all.size() * sizeof(BatchTile), cudaMemcpyHostToDevice, st));
    batch.tile_log = tile_log;
    ntt_batch_set_radix(batch, DV_NTT_RADIX_LOG);
    // the host descriptor vectors must outlive the copies above
    DV_CUDA(cudaStreamSynchronize(st));
}

namespace {
template <int R_LOG>
uint32_t batch_grid(uint32_t ntiles, int tile_log) {
    const int smem = 32 << tile_log;
    // the attribute is a bound shared by every batch: always the largest tile
    DV_CUDA(cudaFuncSetAttribute(k_ntt_batch<R_LOG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 32 << BATCH_TILE_MAX));
    int per_sm = 0;
    DV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ntt_batch<R_LOG>, 256, smem));
    return (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>((uint64_t)sm_count() * (uint32_t)std::max(1, per_sm), ntiles));
}
}  // namespace

void ntt_batch_set_radix(NttBatch& batch, int radix_log) {
    switch (radix_log) {
        case 1: batch.grid = batch_grid<1>(batch.ntiles, batch.tile_log); break;
        case 2: batch.grid = batch_grid<2>(batch.ntiles, batch.tile_log); break;
        case 3: batch.grid = batch_grid<3>(batch.ntiles, batch.tile_log); break;
        default: throw InvalidArgument("batch NTT radix_log must be 1, 2 or 3");
    }
    batch.radix_log = radix_log;
}

void ntt_batch_enqueue(NttBatch& batch, cudaStream_t st) {
    if (!batch.count) return;
    uint32_t* ctl = batch.ctl.as<uint32_t>(2 + 3ull * batch.count);
    DV_CUDA(cudaMemsetAsync(ctl, 0, (2 + 3ull * batch.count) * sizeof(uint32_t), st));
    DV_CUDA(cudaMemsetAsync(batch.errs.as<uint32_t>(batch.count), 0xff, batch.count * sizeof(uint32_t), st));
    const BatchDesc* descs = batch.descs.as<BatchDesc>(batch.count);
    const BatchTile* tiles = batch.tiles.as<BatchTile>(batch.ntiles);
    const int smem = 32 << batch.tile_log;
    switch (batch.radix_log) {
        case 1: k_ntt_batch<1><<<batch.grid, 256, smem, st>>>(descs, tiles, batch.ntiles, ctl); break;
        case 3: k_ntt_batch<3><<<batch.grid, 256, smem, st>>>(descs, tiles, batch.ntiles, ctl); break;
        default: k_ntt_batch<2><<<batch.grid, 256, smem, st>>>(descs, tiles, batch.ntiles, ctl); break;
    }
    DV_LAUNCH();
}

void ntt_batch_check(NttBatch& batch, cudaStream_t st) {
    if (!batch.count) return;
    std::vector<uint32_t> errs(batch.count);
    uint32_t status = 0;
    DV_CUDA(cudaMemcpyAsync(errs.data(), batch.errs.as<uint32_t>(batch.count), batch.count * sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(&status, batch.ctl.as<uint32_t>(2) + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (status) throw CudaFailure("NTT batch: a pass dependency wait timed out");
    for (uint32_t i = 0; i < batch.count; ++i)
        if (errs[i] != 0xffffffffu)
            throw InvalidArgument("non-canonical NTT input in transform " + std::to_string(i) + " at index " +
                                  std::to_string(errs[i]));
}

}  // namespace dv

// =====================================================================
// Allocation-free NTT entry point.
//
// Some callers cannot allocate device memory at the moment they need a
// transform: code that runs while another component owns the allocator
// (a caching allocator or memory pool that must not be bypassed), code
// on a latency-critical path that must never block on cudaMalloc/cudaFree
// (both can synchronise the device), and hosts with a hard device-memory
// budget fixed at start-up.  dvgpu_bn254_ntt_noalloc serves them: the
// caller passes the input and output device buffers and a stream; every
// other buffer the transform needs (the working vector, twiddle and coset
// tables, constants and the error word) lives in the file-scope array
// below, reserved when the library is loaded on a device and kept until
// the process exits.  The array bounds the size: at most 2^16 elements.
//
// The array is shared by all calls on a device and keeps the last call's
// contents; each call rebuilds its tables and resets its error word.  Two
// calls whose work overlaps on the GPU (different streams, no ordering
// between them) race on the array and may both produce wrong results.
// The first call on a device looks up the array's device address; make
// that first call before starting any stream capture.
// =====================================================================
namespace dv {
namespace {

constexpr int NOALLOC_MAX_LOG = 16;
constexpr uint64_t NOALLOC_MAX_N = 1ull << NOALLOC_MAX_LOG;
constexpr uint64_t NOALLOC_TAB = 1ull << ((NOALLOC_MAX_LOG + 1) / 2);
// layout in Fr elements: work | twiddles | coset hi | coset lo | constants | error word
constexpr uint64_t NA_WORK = 0;
constexpr uint64_t NA_TW = NA_WORK + NOALLOC_MAX_N;
constexpr uint64_t NA_HI = NA_TW + NOALLOC_MAX_N / 2;
constexpr uint64_t NA_LO = NA_HI + NOALLOC_TAB;
constexpr uint64_t NA_CONST = NA_LO + NOALLOC_TAB;
constexpr uint64_t NA_ERR = NA_CONST + C_COUNT;
constexpr uint64_t NA_TOTAL = NA_ERR + 1;

static __device__ __align__(256) Fr noalloc_scratch[NA_TOTAL];  // about 3.1 MB per device

constexpr int NOALLOC_MAX_DEVICES = 64;
Fr* noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
cudaError_t noalloc_status[NOALLOC_MAX_DEVICES] = {};
std::once_flag noalloc_once[NOALLOC_MAX_DEVICES];

// Device address of the scratch array on the current device, looked up once
// per device (std::call_once: host threads making their first call on one
// device at the same time wait for a single lookup).  Host code must not use
// the symbol itself as a pointer.  The cached address belongs to the
// device's primary context: it is not valid after cudaDeviceReset.
Fr* noalloc_scratch_on(int dev) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) throw InvalidArgument("device ordinal out of range");
    std::call_once(noalloc_once[dev], [dev] {
        void* p = nullptr;
        noalloc_status[dev] = cudaGetSymbolAddress(&p, noalloc_scratch);
        if (noalloc_status[dev] == cudaSuccess) noalloc_ptr[dev] = static_cast<Fr*>(p);
    });
    DV_CUDA(noalloc_status[dev]);
    return noalloc_ptr[dev];
}

void ntt_noalloc(const uint8_t* d_in, uint8_t* d_out, int logn, int kind, cudaStream_t st) {
    const uint64_t n = 1ull << logn;
    const bool inverse = kind & 1, coset = kind >= 2;
    const int split = (logn + 1) / 2;
    int dev = 0;
    DV_CUDA(cudaGetDevice(&dev));
    Fr* base = noalloc_scratch_on(dev);
    Fr* work = base + NA_WORK;
    Fr* tw = base + NA_TW;
    Fr* hi = base + NA_HI;
    Fr* lo = base + NA_LO;
    Fr* kc = base + NA_CONST;
    uint32_t* bad = reinterpret_cast<uint32_t*>(base + NA_ERR);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), st));
    k_setup_consts<<<1, 1, 0, st>>>(logn, inverse ? 1 : 0, split, kc);
    DV_LAUNCH();
    const uint64_t half = std::max<uint64_t>(1, n / 2);
    const uint32_t chunk = 64;
    const uint64_t threads = (half + chunk - 1) / chunk;
    k_pow_table<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(kc + C_W, nullptr, half, chunk, 0, tw);
    DV_LAUNCH();
    const uint64_t nlo = 1ull << split, nhi = (n + nlo - 1) >> split;
    if (coset) {
        k_pow_table<<<(unsigned)((nhi + 127) / 128), 128, 0, st>>>(inverse ? kc + C_GINV_SPLIT : kc + C_G_SPLIT,
                                                                  inverse ? kc + C_NINV : nullptr, nhi, 1, 0, hi);
        DV_LAUNCH();
        k_pow_table<<<(unsigned)((nlo + 127) / 128), 128, 0, st>>>(inverse ? kc + C_GINV : kc + C_G, nullptr, nlo, 1,
                                                                  0, lo);
        DV_LAUNCH();
    }
    const Fr* pre_hi = (coset && !inverse) ? hi : nullptr;
    const Fr* pre_lo = (coset && !inverse) ? lo : nullptr;
    run_passes(d_in, work, d_out, logn, tw, pre_hi, pre_lo, nullptr, nullptr, nullptr, split, bad, false, st);
    k_permute<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(work, d_out, logn, (coset && inverse) ? hi : nullptr,
                                                          (coset && inverse) ? lo : nullptr, split,
                                                          inverse ? kc + C_NINV : nullptr);
    DV_LAUNCH();
    uint32_t host_bad = 0;
    DV_CUDA(cudaMemcpyAsync(&host_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (host_bad != 0xffffffffu) throw InvalidArgument("non-canonical NTT input at index " + std::to_string(host_bad));
}

}  // namespace
}  // namespace dv

extern "C" int dvgpu_bn254_ntt_noalloc(const uint8_t* d_values, size_t length, int kind, uint8_t* d_result,
                                       void* stream, char* error, size_t error_capacity) {
    auto fail = [&](int status, const std::string& msg) {
        if (error && error_capacity) {
            const size_t k = std::min(error_capacity - 1, msg.size());
            memcpy(error, msg.data(), k);
            error[k] = '\0';
        }
        return status;
    };
    if (!d_values || !d_result || kind < 0 || kind > 3 || !length || (length & (length - 1)))
        return fail(-1, "invalid allocation-free NTT arguments");
    if (length > dv::NOALLOC_MAX_N)
        return fail(-1, "NTT length exceeds the allocation-free maximum of 65536 elements");
    int logn = 0;
    while ((1ull << logn) < length) ++logn;
    try {
        dv::ntt_noalloc(d_values, d_result, logn, kind, static_cast<cudaStream_t>(stream));
        return 0;
    } catch (const dv::InvalidArgument& e) {
        return fail(-1, e.what());
    } catch (const std::exception& e) {
        return fail(-2, e.what());
    } catch (...) {
        return fail(-3, "unknown native exception");
    }
}
