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
// the twiddle's canonical bits taken from the resident Fr twiddle table
// (w^t, t < n/2) and applied by double-and-add; t = 0 skips the product.
// A last launch reads the bit-reversed positions, applies 1/n for the
// inverse and writes canonical affine bytes.
#include <cstring>
#include <string>

#include "abi_util.hpp"
#include "backend.hpp"

namespace dv {
namespace {

// [k] p for a canonical 254-bit scalar k, left to right.
DV_INL XYZZ<Fq> scalar_mul(const XYZZ<Fq>& p, const uint32_t* k) {
    int top = 255;
    while (top >= 0 && !((k[top >> 5] >> (top & 31)) & 1)) --top;
    if (top < 0 || p.is_inf()) return XYZZ<Fq>::inf();
    XYZZ<Fq> r = p;
    for (int i = top - 1; i >= 0; --i) {
        r = XYZZ<Fq>::dbl_paired(r);
        if ((k[i >> 5] >> (i & 31)) & 1) r = XYZZ<Fq>::add_paired(r, p);
    }
    return r;
}

__global__ void k_ec_load(const G1A* __restrict__ conv, uint64_t total, XYZZ<Fq>* __restrict__ work) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    work[i] = XYZZ<Fq>::from_affine(conv[i]);
}

// Stage s of every row: butterfly t of row r pairs positions
// grp * 2 half + pos and that + half, half = n / 2^(s+1).
__global__ void __launch_bounds__(128) k_ec_stage(XYZZ<Fq>* __restrict__ work, int logn, int s, uint64_t butterflies,
                                                  const Fr* __restrict__ tw) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= butterflies) return;
    const uint64_t r = t >> (logn - 1);
    const uint32_t j = (uint32_t)(t & ((1ull << (logn - 1)) - 1));
    const int hlog = logn - 1 - s;
    const uint32_t pos = j & ((1u << hlog) - 1), grp = j >> hlog;
    const uint64_t i0 = (r << logn) + ((uint64_t)grp << (hlog + 1)) + pos, i1 = i0 + (1u << hlog);
    const XYZZ<Fq> a = work[i0], b = work[i1];
    XYZZ<Fq> d = XYZZ<Fq>::add(a, b.neg());
    if (pos) {
        uint32_t k[8];
        tw[(uint64_t)pos << s].to_canonical(k);
        d = scalar_mul(d, k);
    }
    work[i0] = XYZZ<Fq>::add(a, b);
    work[i1] = d;
}

__global__ void __launch_bounds__(128) k_ec_store(const XYZZ<Fq>* __restrict__ work, int logn, uint64_t total,
                                                  const uint32_t* __restrict__ ninv, uint8_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint64_t r = i >> logn;
    const uint32_t e = (uint32_t)(i & ((1ull << logn) - 1));
    const uint32_t src = logn ? (__brev(e) >> (32 - logn)) : 0;
    XYZZ<Fq> p = work[(r << logn) + src];
    if (ninv) {
        uint32_t k[8];
        for (int w = 0; w < 8; ++w) k[w] = ninv[w];
        p = scalar_mul(p, k);
    }
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
    NttTables& tab = ntt_tables(b.ntt, logn, inverse ? NTT_INVERSE : NTT_FORWARD, st);
    const Fr* tw = tab.tw.as<Fr>(1);
    const uint64_t butterflies = total / 2;
    for (int s = 0; s < logn; ++s) {
        k_ec_stage<<<(unsigned)((butterflies + 127) / 128), 128, 0, st>>>(work, logn, s, butterflies, tw);
        DV_LAUNCH();
    }
    k_ec_store<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(work, logn, total,
                                                                inverse ? ntt_ninv_canonical(tab) : nullptr, d_out);
    DV_LAUNCH();
}

// Bit-reversed XYZZ working rows -> natural-order XYZZ rows (x 1/n).
__global__ void __launch_bounds__(128) k_ec_permute(const XYZZ<Fq>* __restrict__ work, int logn, uint64_t total,
                                                    const uint32_t* __restrict__ ninv, XYZZ<Fq>* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint64_t r = i >> logn;
    const uint32_t e = (uint32_t)(i & ((1ull << logn) - 1));
    const uint32_t src = logn ? (__brev(e) >> (32 - logn)) : 0;
    XYZZ<Fq> p = work[(r << logn) + src];
    if (ninv) {
        uint32_t k[8];
        for (int w = 0; w < 8; ++w) k[w] = ninv[w];
        p = scalar_mul(p, k);
    }
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
    NttTables& tab = ntt_tables(ws, logn, inverse ? NTT_INVERSE : NTT_FORWARD, st);
    const Fr* tw = tab.tw.as<Fr>(1);
    const uint64_t butterflies = total / 2;
    for (int s = 0; s < logn; ++s) {
        k_ec_stage<<<(unsigned)((butterflies + 127) / 128), 128, 0, st>>>(work, logn, s, butterflies, tw);
        DV_LAUNCH();
    }
    k_ec_permute<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(work, logn, total,
                                                                  inverse ? ntt_ninv_canonical(tab) : nullptr, out);
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
