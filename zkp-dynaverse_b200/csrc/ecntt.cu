// G1 transform (EC-NTT): rows of G1 points through the radix-2 FFT of the
// Fr domain, the group action of the twiddles standing in for the field
// product.
//
// Semantics of RebuildBackend::transform_rows with kind G1
// (crates/protocol/src/incremental_rebuild/operators.rs:413-440, arkworks
// Radix2EvaluationDomain::fft_in_place / ifft_in_place over G1Projective):
// per row of n = 2^k points, out_i = sum_j w^(ij) P_j in natural order with
// w the arkworks root of order n; the inverse uses w^-1 and scales by 1/n;
// each row is normalised to affine.  The reference's GPU form is ICICLE's
// dvgpu_ecntt_rows (native/src/icicle_ntt.cu:90-95).
//
// Layout: points in XYZZ form (128 bytes) in a working vector; one launch
// per decimation-in-frequency stage, one thread per butterfly
//      (a, b) -> (a + b, [w^t] (a - b)),
// t = 0 skipping the product.  A last launch reads the bit-reversed
// positions, applies 1/n for the inverse and writes canonical affine bytes.
//
// Scalar multiplications use the GLV endomorphism of BN254 G1 (Gallant,
// Lambert, Vanstone, CRYPTO 2001): phi(x, y) = (beta x, y) = [lambda] P with
// beta, lambda cube roots of unity.  Each twiddle k = w^t is split once per
// table into k = k1 + k2 lambda (mod r), |k1|, |k2| < 2^128, by rounding
// against the short lattice basis (a1, b1) = (9931322734385697763,
// -147946756881789319000765030803803410728), (a2, b2) =
// (147946756881789319010696353538189108491, 9931322734385697763):
//   c1 = (k g1) >> 256, c2 = (k g2) >> 256, g1 = round(2^256 b2 / r),
//   g2 = round(-2^256 b1 / r), k1 = k - c1 a1 - c2 a2, k2 = -c1 b1 - c2 b2.
// [k] P = [k1] P + [k2] phi(P) by one joint double-and-add over the longer
// half (about 127 doublings and 96 additions instead of 254 and 127).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "abi_util.hpp"
#include "backend.hpp"

namespace dv {
namespace {

// A scalar split for GLV: |k1|, |k2| (little-endian words), sign flags (bit
// 0: k1 < 0, bit 1: k2 < 0) and the bit length of the longer half.
struct __align__(16) GlvScalar {
    uint32_t k1[4], k2[4];
    uint32_t flags, bits, pad[2];
};

// beta (Montgomery): phi(x, y) = (beta x, y) = [lambda] (x, y) on G1.
__device__ __constant__ uint32_t GLV_BETA[8] = {0xd782e155u, 0x71930c11u, 0xffbe3323u, 0xa6bb947cu,
                                                0xd4741444u, 0xaa303344u, 0x26594943u, 0x2c3b3f0du};

// [k] p = [k1] p + [k2] phi(p) over signed fixed windows of 5 bits: both
// halves recoded into digits in [-16, 16) (k = sum d_j 32^j, at most 26
// windows for halves below 2^128), one table of |d| p for |d| = 1..16 (8
// doublings and 7 additions, in local memory) serving both halves, the
// second through phi (one product: beta X).  Every lane of a warp adds at
// the same window positions, so a warp runs 5 doublings and 2 additions a
// window; a sparse signed-digit form would make each warp add wherever any
// of its lanes has a digit, nearly every bit.
DV_INL void recode5(const uint32_t* k, int nw, int8_t* d) {
    uint32_t carry = 0;
    for (int j = 0; j < nw; ++j) {
        const int b = 5 * j, w = b >> 5, sh = b & 31;
        uint32_t x = k[w] >> sh;
        if (sh > 27 && w + 1 < 4) x |= k[w + 1] << (32 - sh);
        const int v = (int)((x & 31u) + carry);
        carry = v >= 16 ? 1u : 0u;
        d[j] = (int8_t)(v >= 16 ? v - 32 : v);
    }
}
DV_INL XYZZ<Fq> scalar_mul(const XYZZ<Fq>& p, const GlvScalar& g) {
    if (p.is_inf() || g.bits == 0) return XYZZ<Fq>::inf();
    Fq beta;
#pragma unroll
    for (int i = 0; i < 8; ++i) beta.v[i] = GLV_BETA[i];
    // the top window holds at most 3 bits, so the recoding's carry never leaves it
    const int nw = ((int)g.bits + 1) / 5 + 1;
    int8_t d1[26], d2[26];
    recode5(g.k1, nw, d1);
    recode5(g.k2, nw, d2);
    XYZZ<Fq> tab[16];
    tab[0] = p;
#pragma unroll 1
    for (int m = 2; m <= 16; ++m)
        tab[m - 1] = (m & 1) ? XYZZ<Fq>::add_paired(tab[m - 2], p) : XYZZ<Fq>::dbl_paired(tab[m / 2 - 1]);
    const bool n1 = g.flags & 1, n2 = g.flags & 2;
    XYZZ<Fq> r = XYZZ<Fq>::inf();
#pragma unroll 1
    for (int j = nw - 1; j >= 0; --j) {
        if (j != nw - 1)
#pragma unroll 1
            for (int i = 0; i < 5; ++i) r = XYZZ<Fq>::dbl_paired(r);
        const int a = d1[j], b = d2[j];
        if (a) {
            const XYZZ<Fq> t = tab[(a < 0 ? -a : a) - 1];
            r = XYZZ<Fq>::add_paired(r, (a < 0) != n1 ? t.neg() : t);
        }
        if (b) {
            XYZZ<Fq> t = tab[(b < 0 ? -b : b) - 1];
            t.x = Fq::mul(t.x, beta);
            r = XYZZ<Fq>::add_paired(r, (b < 0) != n2 ? t.neg() : t);
        }
    }
    return r;
}

// ---- host: the GLV split of canonical scalars (4 x 64-bit words)
typedef unsigned __int128 u128;
struct W4 {
    uint64_t w[4];
};
constexpr uint64_t GLV_A1 = 9931322734385697763ull;                                  // = b2
const W4 GLV_B1ABS = {{0x8211bbeb7d4f1128ull, 0x6f4d8248eeb859fcull, 0, 0}};      // -b1
const W4 GLV_A2 = {{0x0be4e1541221250bull, 0x6f4d8248eeb859fdull, 0, 0}};
const W4 GLV_G1 = {{0xd91d232ec7e0b3d7ull, 0x2ull, 0, 0}};
const W4 GLV_G2 = {{0x7a7bd9d4391eb18eull, 0x4ccef014a773d2cfull, 0x2ull, 0}};

// (a b) mod 2^256 and (a b) >> 256
void mul_w4(const W4& a, const W4& b, W4* lo, W4* hi) {
    uint64_t t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
        u128 c = 0;
        for (int j = 0; j < 4; ++j) {
            c += (u128)a.w[i] * b.w[j] + t[i + j];
            t[i + j] = (uint64_t)c;
            c >>= 64;
        }
        t[i + 4] = (uint64_t)c;
    }
    if (lo) for (int i = 0; i < 4; ++i) lo->w[i] = t[i];
    if (hi) for (int i = 0; i < 4; ++i) hi->w[i] = t[i + 4];
}
W4 sub_w4(const W4& a, const W4& b) {
    W4 r;
    uint64_t borrow = 0;
    for (int i = 0; i < 4; ++i) {
        const u128 d = (u128)a.w[i] - b.w[i] - borrow;
        r.w[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    return r;
}
// |x| of a two's complement 256-bit value, into 4 x 32-bit words; false if >= 2^128
bool magnitude(const W4& x, uint32_t* out, bool* negative) {
    W4 m = x;
    *negative = (x.w[3] >> 63) != 0;
    if (*negative) m = sub_w4(W4{{0, 0, 0, 0}}, x);
    if (m.w[2] || m.w[3]) return false;
    out[0] = (uint32_t)m.w[0]; out[1] = (uint32_t)(m.w[0] >> 32);
    out[2] = (uint32_t)m.w[1]; out[3] = (uint32_t)(m.w[1] >> 32);
    return true;
}
int bit_length(const uint32_t* w) {
    for (int i = 127; i >= 0; --i)
        if ((w[i >> 5] >> (i & 31)) & 1) return i + 1;
    return 0;
}
GlvScalar glv_split(const uint64_t* k_words) {
    const W4 k = {{k_words[0], k_words[1], k_words[2], k_words[3]}};
    W4 c1, c2, t1, t2;
    mul_w4(k, GLV_G1, nullptr, &c1);
    mul_w4(k, GLV_G2, nullptr, &c2);
    mul_w4(c1, W4{{GLV_A1, 0, 0, 0}}, &t1, nullptr);
    mul_w4(c2, GLV_A2, &t2, nullptr);
    const W4 k1 = sub_w4(sub_w4(k, t1), t2);  // k - c1 a1 - c2 a2
    mul_w4(c1, GLV_B1ABS, &t1, nullptr);
    mul_w4(c2, W4{{GLV_A1, 0, 0, 0}}, &t2, nullptr);
    const W4 k2 = sub_w4(t1, t2);             // -c1 b1 - c2 b2
    GlvScalar g{};
    bool n1, n2;
    if (!magnitude(k1, g.k1, &n1) || !magnitude(k2, g.k2, &n2)) throw CudaFailure("GLV split out of range");
    g.flags = (n1 ? 1u : 0u) | (n2 ? 2u : 0u);
    g.bits = (uint32_t)std::max(bit_length(g.k1), bit_length(g.k2));
    return g;
}

__global__ void k_tw_canonical(const Fr* __restrict__ tw, uint64_t n, Fr* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr one_raw = Fr::zero();
    one_raw.v[0] = 1;
    out[i] = Fr::mul(tw[i], one_raw);
}

// GLV splits of the table's n/2 twiddles, then of 1/n (inverse tables), built
// once per (size, direction) and kept with the twiddles.
const GlvScalar* glv_table(NttWorkspace& ws, int logn, bool inverse, cudaStream_t st) {
    NttTables& tab = ntt_tables(ws, logn, inverse ? NTT_INVERSE : NTT_FORWARD, st);
    const uint64_t half = (1ull << logn) / 2;
    if (tab.glv_ready) return tab.glv.view<GlvScalar>();
    std::vector<uint64_t> words(4 * (half + 1), 0);
    if (half) {
        DevBuf canon;
        Fr* c = canon.as<Fr>(half);
        k_tw_canonical<<<(unsigned)((half + 127) / 128), 128, 0, st>>>(tab.tw.as<Fr>(1), half, c);
        DV_LAUNCH();
        DV_CUDA(cudaMemcpyAsync(words.data(), c, 32 * half, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    }
    if (inverse) {
        DV_CUDA(cudaMemcpyAsync(words.data() + 4 * half, ntt_ninv_canonical(tab), 32, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<GlvScalar> table(half + 1);
    for (uint64_t i = 0; i <= half; ++i) table[i] = glv_split(words.data() + 4 * i);
    GlvScalar* d = tab.glv.as<GlvScalar>(half + 1);
    DV_CUDA(cudaMemcpyAsync(d, table.data(), sizeof(GlvScalar) * (half + 1), cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaStreamSynchronize(st));
    tab.glv_ready = 1;
    return d;
}

__global__ void k_ec_load(const G1A* __restrict__ conv, uint64_t total, XYZZ<Fq>* __restrict__ work) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    work[i] = XYZZ<Fq>::from_affine(conv[i]);
}

// Stage s of every row: butterfly t of row r pairs positions
// grp * 2 half + pos and that + half, half = n / 2^(s+1).
__global__ void __launch_bounds__(128) k_ec_stage(XYZZ<Fq>* __restrict__ work, int logn, int s, uint64_t butterflies,
                                                  const GlvScalar* __restrict__ tw) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= butterflies) return;
    const uint64_t r = t >> (logn - 1);
    const uint32_t j = (uint32_t)(t & ((1ull << (logn - 1)) - 1));
    const int hlog = logn - 1 - s;
    const uint32_t pos = j & ((1u << hlog) - 1), grp = j >> hlog;
    const uint64_t i0 = (r << logn) + ((uint64_t)grp << (hlog + 1)) + pos, i1 = i0 + (1u << hlog);
    const XYZZ<Fq> a = work[i0], b = work[i1];
    XYZZ<Fq> d = XYZZ<Fq>::add(a, b.neg());
    if (pos) d = scalar_mul(d, tw[(uint64_t)pos << s]);
    work[i0] = XYZZ<Fq>::add(a, b);
    work[i1] = d;
}

__global__ void __launch_bounds__(128) k_ec_store(const XYZZ<Fq>* __restrict__ work, int logn, uint64_t total,
                                                  const GlvScalar* __restrict__ ninv, uint8_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint64_t r = i >> logn;
    const uint32_t e = (uint32_t)(i & ((1ull << logn) - 1));
    const uint32_t src = logn ? (__brev(e) >> (32 - logn)) : 0;
    XYZZ<Fq> p = work[(r << logn) + src];
    if (ninv) p = scalar_mul(p, *ninv);
    uint8_t* o = out + 64 * i;
    if (p.is_inf()) {
        const uint4 z = make_uint4(0, 0, 0, 0);
        for (int b = 0; b < 64; b += 16) *reinterpret_cast<uint4*>(o + b) = z;
        return;
    }
    const G1A a = p.to_affine();
    store_canonical(o, a.x);
    store_canonical(o + 32, a.y);
}

// Transforms rows x 2^logn canonical G1 points (device) into d_out.
void g1_ntt_rows(Backend& b, const uint8_t* d_in, int logn, uint64_t rows, bool inverse, uint8_t* d_out,
                 cudaStream_t st) {
    const uint64_t n = 1ull << logn, total = n * rows;
    G1A* conv = b.conv_points.as<G1A>(total);
    uint32_t* bad = b.err.as<uint32_t>(1);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), st));
    convert_points<Fq>(d_in, conv, total, bad, st);
    const uint32_t first_bad = read_err_word(b, bad, st);
    if (first_bad != 0xffffffffu) throw InvalidArgument("invalid point at index " + std::to_string(first_bad));
    XYZZ<Fq>* work = b.aux.as<XYZZ<Fq>>(total);
    k_ec_load<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(conv, total, work);
    DV_LAUNCH();
    const GlvScalar* tw = glv_table(b.ntt, logn, inverse, st);
    const uint64_t butterflies = total / 2;
    for (int s = 0; s < logn; ++s) {
        k_ec_stage<<<(unsigned)((butterflies + 127) / 128), 128, 0, st>>>(work, logn, s, butterflies, tw);
        DV_LAUNCH();
    }
    k_ec_store<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(work, logn, total,
                                                                inverse ? tw + (1ull << logn) / 2 : nullptr, d_out);
    DV_LAUNCH();
}

// Bit-reversed XYZZ working rows -> natural-order XYZZ rows (x 1/n).
__global__ void __launch_bounds__(128) k_ec_permute(const XYZZ<Fq>* __restrict__ work, int logn, uint64_t total,
                                                    const GlvScalar* __restrict__ ninv, XYZZ<Fq>* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint64_t r = i >> logn;
    const uint32_t e = (uint32_t)(i & ((1ull << logn) - 1));
    const uint32_t src = logn ? (__brev(e) >> (32 - logn)) : 0;
    XYZZ<Fq> p = work[(r << logn) + src];
    if (ninv) p = scalar_mul(p, *ninv);
    out[i] = p;
}

int log2_exact(uint64_t n) {
    int k = 0;
    while ((1ull << k) < n) ++k;
    return (1ull << k) == n ? k : -1;
}

}  // namespace

void g1_ntt_rows_xyzz(NttWorkspace& ws, XYZZ<Fq>* work, int logn, uint64_t rows, bool inverse, XYZZ<Fq>* out,
                      cudaStream_t st) {
    const uint64_t total = rows << logn;
    const GlvScalar* tw = glv_table(ws, logn, inverse, st);
    const uint64_t butterflies = total / 2;
    for (int s = 0; s < logn; ++s) {
        k_ec_stage<<<(unsigned)((butterflies + 127) / 128), 128, 0, st>>>(work, logn, s, butterflies, tw);
        DV_LAUNCH();
    }
    k_ec_permute<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(work, logn, total,
                                                                  inverse ? tw + (1ull << logn) / 2 : nullptr, out);
    DV_LAUNCH();
}

}  // namespace dv

using namespace dv;

extern "C" int dvgpu_bn254_g1_ntt_rows_device(void* opaque, const uint8_t* d_points, size_t row_len, size_t rows,
                                              int inverse, uint8_t* d_results, void* stream, char* error,
                                              size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        const int logn = log2_exact(row_len);
        require(logn >= 0 && logn <= 20 && rows >= 1 && row_len * rows <= (1ull << 24),
                "G1 transform rows must be 1..2^20 points (a power of two), at most 2^24 points in all");
        require(d_points && d_results && (inverse == 0 || inverse == 1), "invalid G1 transform arguments");
        const cudaStream_t st = pick(b, stream);
        g1_ntt_rows(b, d_points, logn, rows, inverse, d_results, st);
        DV_CUDA(cudaStreamSynchronize(st));
    });
}

extern "C" int dvgpu_bn254_g1_ntt_rows(void* opaque, const uint8_t* points, size_t row_len, size_t rows, int inverse,
                                       uint8_t* results, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        const int logn = log2_exact(row_len);
        require(logn >= 0 && logn <= 20 && rows >= 1 && row_len * rows <= (1ull << 24),
                "G1 transform rows must be 1..2^20 points (a power of two), at most 2^24 points in all");
        require(points && results && (inverse == 0 || inverse == 1), "invalid G1 transform arguments");
        const uint64_t total = (uint64_t)row_len * rows;
        uint8_t* d_in = b.in_points.as<uint8_t>(64 * total);
        uint8_t* d_out = b.out_buf.as<uint8_t>(64 * total);
        DV_CUDA(cudaMemcpyAsync(d_in, points, 64 * total, cudaMemcpyHostToDevice, b.stream));
        g1_ntt_rows(b, d_in, logn, rows, inverse, d_out, b.stream);
        DV_CUDA(cudaMemcpyAsync(results, d_out, 64 * total, cudaMemcpyDeviceToHost, b.stream));
        DV_CUDA(cudaStreamSynchronize(b.stream));
    });
}
