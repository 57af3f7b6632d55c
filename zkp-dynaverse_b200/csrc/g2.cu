// G2 validation and fixed-base generation kernels (see g2.cuh).
#include "g2.cuh"

namespace dv {

namespace {

// psi constants xi^((q-1)/3), xi^((q-1)/2), xi = 9 + u (canonical limbs).
__device__ __constant__ uint32_t PSI_C[4][8] = {
    {0x176f553du, 0x99e39557u, 0xc2c3330cu, 0xb78cc310u, 0xf559b143u, 0x4c0bec3cu, 0x4f7911f7u, 0x2fb34798u},
    {0x640fcba2u, 0x1665d51cu, 0x0b7c9dceu, 0x32ae2a1du, 0xd75a0794u, 0x4ba4cc8bu, 0x61ebae20u, 0x16c9e550u},
    {0x71a0135au, 0xdc540146u, 0xa9c95998u, 0xdbaae0edu, 0xb6e2f9b9u, 0xdc5ec698u, 0x489af5dcu, 0x063cf305u},
    {0x2623b0e3u, 0x82d37f63u, 0x8fa25bd2u, 0x21807dc9u, 0xec796f2bu, 0x0704b5a7u, 0xac41049au, 0x07c03cbcu}};

// r (the group order) as an integer, and the multipliers of algorithms 2/3.
__device__ __constant__ uint32_t R_INT[8] = {0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u,
                                             0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
__device__ __constant__ uint32_t LAMBDA[4] = {0xe87cfd46u, 0xf83e9682u, 0xeeb859fbu, 0x6f4d8248u};  // 6 x^2
__device__ __constant__ uint32_t SEED[2] = {0x4a6909f1u, 0x44e992b4u};                               // x

DV_INL Fq2 psi_cx() {
    uint32_t a[8], b[8];
    for (int i = 0; i < 8; ++i) { a[i] = PSI_C[0][i]; b[i] = PSI_C[1][i]; }
    return {Fq::from_canonical(a), Fq::from_canonical(b)};
}
DV_INL Fq2 psi_cy() {
    uint32_t a[8], b[8];
    for (int i = 0; i < 8; ++i) { a[i] = PSI_C[2][i]; b[i] = PSI_C[3][i]; }
    return {Fq::from_canonical(a), Fq::from_canonical(b)};
}

DV_INL G2X psi(const G2X& p, const Fq2& cx, const Fq2& cy) {
    if (p.is_inf()) return p;
    return {Fq2::mul(Fq2::conj(p.x), cx), Fq2::mul(Fq2::conj(p.y), cy), Fq2::conj(p.zz), Fq2::conj(p.zzz)};
}

template <int WORDS>
DV_INL G2X mul_int(const G2A& a, const uint32_t* k, int bits) {
    G2X r = G2X::inf();
    for (int i = bits - 1; i >= 0; --i) {
        r = G2X::dbl(r);
        if ((k[i >> 5] >> (i & 31)) & 1) r = G2X::add_affine(r, a);
    }
    return r;
}

// Returns the reference mask (0 / 1 / 2 / 4).  One instantiation per
// subgroup algorithm: each kernel then holds only its own algorithm's live
// values (a single kernel with a runtime branch took the registers of the
// largest and spilled).
template <int ALG>
DV_INL uint32_t g2_wire_check(const uint8_t* b) {
    uint32_t w[4][8];
    uint32_t any = 0;
    for (int j = 0; j < 4; ++j) {
        load_words(b + 32 * j, w[j]);
        for (int i = 0; i < 8; ++i) any |= w[j][i];
    }
    if (!any) return 0;
    const uint32_t flags = (w[3][7] >> 24) & 0xc0u;
    if (flags == 0xc0u) return 1;
    w[3][7] &= 0x3fffffffu;
    for (int j = 0; j < 4; ++j)
        if (!Fq::is_canonical(w[j])) return 1;
    if (flags == 0x40u) return 0;
    G2A p;
    p.x = {Fq::from_canonical(w[0]), Fq::from_canonical(w[1])};
    p.y = {Fq::from_canonical(w[2]), Fq::from_canonical(w[3])};
    // (0, 0) with the 0x80 flag is a parsed point, not infinity: test the
    // equation directly (0 = b' fails, as in the reference parser).
    if (!(Fq2::sqr(p.y) == Fq2::add(Fq2::mul(Fq2::sqr(p.x), p.x), g2_b()))) return 2;
    bool ok;
    if constexpr (ALG == 1) {
        uint32_t r[8];
        for (int i = 0; i < 8; ++i) r[i] = R_INT[i];
        ok = mul_int<8>(p, r, 254).is_inf();
    } else if constexpr (ALG == 2) {
        uint32_t l[4];
        for (int i = 0; i < 4; ++i) l[i] = LAMBDA[i];
        const G2X lhs = psi(G2X::from_affine(p), psi_cx(), psi_cy());
        ok = G2X::equal(lhs, mul_int<4>(p, l, 127));
    } else {
        // [x]P + psi([x]P) + psi^2([x]P) + P == 2 psi^3([x]P), each point
        // folded into the left side as soon as the next is formed, and the
        // psi constants read from constant memory where used, so at most two
        // projective points are live at once
        uint32_t s[2] = {SEED[0], SEED[1]};
        G2X t = mul_int<2>(p, s, 63);
        G2X lhs = G2X::add_affine(t, p);
        t = psi(t, psi_cx(), psi_cy());
        lhs = G2X::add(lhs, t);
        t = psi(t, psi_cx(), psi_cy());
        lhs = G2X::add(lhs, t);
        t = G2X::dbl(psi(t, psi_cx(), psi_cy()));
        ok = G2X::equal(lhs, t);
    }
    return ok ? 0 : 4;
}

template <int ALG>
__global__ void __launch_bounds__(256) k_g2_check(const uint8_t* __restrict__ wire, uint64_t n,
                                                  uint32_t* __restrict__ masks, G2CheckAccum* __restrict__ acc) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t m = g2_wire_check<ALG>(wire + 128 * i);
    masks[i] = m;
    if (m) {
        atomicAdd(&acc->invalid, 1ull);
        atomicMin(&acc->first, (unsigned long long)i);
        atomicOr(&acc->mask, m);
    }
}

// ------------------------------------------------------------------ fixed base
template <class F>
DV_INL Affine<F> generator();
template <>
DV_INL Affine<Fq> generator<Fq>() {
    uint32_t x[8] = {1, 0, 0, 0, 0, 0, 0, 0}, y[8] = {2, 0, 0, 0, 0, 0, 0, 0};
    return {Fq::from_canonical(x), Fq::from_canonical(y)};
}
// Standard BN254 G2 generator (ark-bn254 0.4.0), canonical limbs.
__device__ __constant__ uint32_t G2_GEN[4][8] = {
    {0xd992f6edu, 0x46debd5cu, 0xf75edaddu, 0x674322d4u, 0x5e5c4479u, 0x426a0066u, 0x121f1e76u, 0x1800deefu},
    {0xaef312c2u, 0x97e485b7u, 0x35a9e712u, 0xf1aa4933u, 0x31fb5d25u, 0x7260bfb7u, 0x920d483au, 0x198e9393u},
    {0x66fa7daau, 0x4ce6cc01u, 0x0c43d37bu, 0xe3d1e769u, 0x8dcb408fu, 0x4aab7180u, 0xdb8c6debu, 0x12c85ea5u},
    {0xd122975bu, 0x55acdadcu, 0x70b38ef3u, 0xbc4b3133u, 0x690c3395u, 0xec9e99adu, 0x585ff075u, 0x090689d0u}};
template <>
DV_INL Affine<Fq2> generator<Fq2>() {
    uint32_t w[4][8];
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 8; ++i) w[j][i] = G2_GEN[j][i];
    return {{Fq::from_canonical(w[0]), Fq::from_canonical(w[1])}, {Fq::from_canonical(w[2]), Fq::from_canonical(w[3])}};
}

// Fixed-base tables: scalars as 16 signed digits of 16 bits,
// s = sum d_w 2^(16 w) with d_w in [-2^15, 2^15) (s < r < 2^254, so the top
// digit takes the last carry), and table[w 2^15 + |d| - 1] = |d| 2^(16 w) G
// in affine Montgomery form: 2^19 entries, 32 MB for G1 and 64 MB for G2,
// built once per backend and read from L2.  A scalar then costs 16 mixed
// additions.
constexpr int FB_WINDOWS = 16;
constexpr uint32_t FB_HALF = 1u << 15;
constexpr uint32_t FB_RUN = 16;  // table entries per build thread

// bases[w] = 2^(16 w) G, one thread per window.
template <class F>
__global__ void k_fb_bases(XYZZ<F>* __restrict__ bases) {
    const int w = threadIdx.x;
    if (w >= FB_WINDOWS) return;
    XYZZ<F> b = XYZZ<F>::from_affine(generator<F>());
    for (int k = 0; k < 16 * w; ++k) b = XYZZ<F>::dbl(b);
    bases[w] = b;
}

// Thread t of window w builds entries j0 .. j0 + 15 (j0 = 16 (t mod 2^11)):
// (j0 + 1) B by double-and-add, then B added per entry; every entry is
// normalised by a warp-wide inversion (all lanes run the same 16 steps).
template <class F>
__global__ void __launch_bounds__(128) k_fb_table(const XYZZ<F>* __restrict__ bases, Affine<F>* __restrict__ table) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;  // grid covers exactly 16 * 2^11 threads
    const uint32_t per_w = FB_HALF / FB_RUN;
    const uint32_t w = t / per_w, j0 = (t % per_w) * FB_RUN;
    const XYZZ<F> b = bases[w];
    XYZZ<F> p = XYZZ<F>::inf();
    const uint32_t m = j0 + 1;
    for (int bit = 15; bit >= 0; --bit) {
        p = XYZZ<F>::dbl(p);
        if ((m >> bit) & 1u) p = XYZZ<F>::add(p, b);
    }
    for (uint32_t e = 0; e < FB_RUN; ++e) {
        const bool inf = p.is_inf();
        const F d = warp_batch_inverse<F>(inf ? F::one() : F::mul(p.zz, p.zzz));
        Affine<F> a = Affine<F>::inf();
        if (!inf) a = {F::mul(p.x, F::mul(d, p.zzz)), F::mul(p.y, F::mul(d, p.zz))};
        table[(size_t)w * FB_HALF + j0 + e] = a;
        p = XYZZ<F>::add(p, b);
    }
}

template <class F>
__global__ void __launch_bounds__(128) k_fb_generate(const uint8_t* __restrict__ scalars, uint64_t n,
                                                     const Affine<F>* __restrict__ table, uint8_t* __restrict__ out,
                                                     uint32_t* __restrict__ first_bad) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    XYZZ<F> acc = XYZZ<F>::inf();
    if (active) {
        uint32_t s[8];
        load_words(scalars + 32 * i, s);
        if (!Fr::is_canonical(s)) {
            atomicMin(first_bad, (uint32_t)i);
        } else {
            uint32_t carry = 0;
#pragma unroll 1
            for (int w = 0; w < FB_WINDOWS; ++w) {
                const uint32_t v = ((s[w >> 1] >> (16 * (w & 1))) & 0xffffu) + carry;
                carry = v >= FB_HALF ? 1u : 0u;
                const int d = carry ? (int)v - (int)(2 * FB_HALF) : (int)v;
                if (d) {
                    Affine<F> e = table[(size_t)w * FB_HALF + (uint32_t)(d < 0 ? -d : d) - 1];
                    if (d < 0) e.y = F::neg(e.y);
                    acc = XYZZ<F>::add_affine(acc, e);
                }
            }
        }
    }
    // all lanes take part in the warp inversion; infinity contributes 1
    const bool inf = acc.is_inf();
    const F den = inf ? F::one() : F::mul(acc.zz, acc.zzz);
    const F d = warp_batch_inverse<F>(den);
    if (!active) return;
    const size_t bytes = 2 * sizeof(F);
    uint8_t* o = out + bytes * i;
    if (inf) {
        for (size_t k = 0; k < bytes; k += 16) *reinterpret_cast<uint4*>(o + k) = make_uint4(0, 0, 0, 0);
        return;
    }
    const F x = F::mul(acc.x, F::mul(d, acc.zzz));
    const F y = F::mul(acc.y, F::mul(d, acc.zz));
    store_canonical(o, x);
    store_canonical(o + sizeof(F), y);
}

inline unsigned blocks_for(uint64_t n, unsigned threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

void g2_check_launch(const uint8_t* d_wire, uint64_t n, uint32_t algorithm, uint32_t* d_masks, G2CheckAccum* d_acc,
                     cudaStream_t st, unsigned threads) {
    if (!n) return;
    // algorithm 3 unless 1 or 2 (the reference's selection)
    if (algorithm == 1) k_g2_check<1><<<blocks_for(n, threads), threads, 0, st>>>(d_wire, n, d_masks, d_acc);
    else if (algorithm == 2) k_g2_check<2><<<blocks_for(n, threads), threads, 0, st>>>(d_wire, n, d_masks, d_acc);
    else k_g2_check<3><<<blocks_for(n, threads), threads, 0, st>>>(d_wire, n, d_masks, d_acc);
    DV_LAUNCH();
}

void g2_kernel_resources(unsigned threads, DvgpuG2KernelResources& out) {
    int dev = 0, max_threads = 0, blocks = 0, nblocks = 0;
    DV_CUDA(cudaGetDevice(&dev));
    DV_CUDA(cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
    cudaFuncAttributes a{}, na{};
    DV_CUDA(cudaFuncGetAttributes(&a, k_g2_check<3>));  // the default algorithm's kernel
    DV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_g2_check<3>, (int)threads, 0));
    // the checked fixed-base normalisation is fused into its generation kernel
    DV_CUDA(cudaFuncGetAttributes(&na, k_fb_generate<Fq2>));
    DV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nblocks, k_fb_generate<Fq2>, 128, 0));
    out = {};
    out.registers = (uint32_t)a.numRegs;
    out.block_threads = threads;
    out.active_blocks = (uint32_t)blocks;
    out.max_threads_per_sm = (uint32_t)max_threads;
    out.local_bytes = a.localSizeBytes;
    out.shared_bytes = a.sharedSizeBytes;
    out.normalize_registers = (uint32_t)na.numRegs;
    out.normalize_active_blocks = (uint32_t)nblocks;
    out.normalize_local_bytes = na.localSizeBytes;
    out.normalize_shared_bytes = na.sharedSizeBytes;
}

namespace {
__global__ void k_fb_validate(const uint8_t* __restrict__ scalars, uint64_t n, uint32_t* __restrict__ first_bad) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s[8];
    load_words(scalars + 32 * i, s);
    if (!Fr::is_canonical(s)) atomicMin(first_bad, (uint32_t)i);
}
}  // namespace

void fixed_base_validate(const uint8_t* d_scalars, uint64_t n, uint32_t* d_first_bad, cudaStream_t st) {
    if (!n) return;
    k_fb_validate<<<blocks_for(n, 256), 256, 0, st>>>(d_scalars, n, d_first_bad);
    DV_LAUNCH();
}

uint64_t fixed_base_table_entries() { return (uint64_t)FB_WINDOWS * FB_HALF; }

void fixed_base_launch(FixedBaseTables& tabs, const uint8_t* d_scalars, uint64_t n, int g2, uint8_t* d_out,
                       uint32_t* d_first_bad, cudaStream_t st) {
    if (!n) return;
    const uint64_t entries = (uint64_t)FB_WINDOWS * FB_HALF;
    const unsigned build_blocks = (unsigned)(entries / FB_RUN / 128);
    if (g2) {
        G2A* t = tabs.g2.as<G2A>(entries);
        if (!tabs.g2_ready) {
            G2X* bases = tabs.bases.as<G2X>(FB_WINDOWS);
            k_fb_bases<Fq2><<<1, 32, 0, st>>>(bases);
            DV_LAUNCH();
            k_fb_table<Fq2><<<build_blocks, 128, 0, st>>>(bases, t);
            DV_LAUNCH();
            tabs.g2_ready = true;
        }
        k_fb_generate<Fq2><<<blocks_for(n, 128), 128, 0, st>>>(d_scalars, n, t, d_out, d_first_bad);
    } else {
        G1A* t = tabs.g1.as<G1A>(entries);
        if (!tabs.g1_ready) {
            G1X* bases = tabs.bases.as<G1X>(FB_WINDOWS);
            k_fb_bases<Fq><<<1, 32, 0, st>>>(bases);
            DV_LAUNCH();
            k_fb_table<Fq><<<build_blocks, 128, 0, st>>>(bases, t);
            DV_LAUNCH();
            tabs.g1_ready = true;
        }
        k_fb_generate<Fq><<<blocks_for(n, 128), 128, 0, st>>>(d_scalars, n, t, d_out, d_first_bad);
    }
    DV_LAUNCH();
}

}  // namespace dv
