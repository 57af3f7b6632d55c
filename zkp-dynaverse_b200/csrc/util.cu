// Seeded synthetic inputs generated on the device (benchmark workloads):
// uniform Fr scalars by rejection sampling of 254-bit words from a
// counter-based hash (splitmix64 finaliser, Steele, Lea, Flood 2014), and
// the powers tau^i of a scalar (an SRS exponent vector) by a chunked
// power table.
#include "curve.cuh"
#include "engine.hpp"

namespace dv {

uint64_t& launch_counter() {
    static uint64_t counter = 0;
    return counter;
}

uint64_t& alloc_counter() {
    static uint64_t counter = 0;
    return counter;
}

uint64_t& alloc_ns_counter() {
    static uint64_t counter = 0;
    return counter;
}

uint64_t* slowest_alloc() {
    static uint64_t record[3] = {0, 0, 0};
    return record;
}

namespace {

DV_INL uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void k_random_fr(uint64_t seed, uint64_t n, uint32_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t w[8];
    for (uint32_t attempt = 0;; ++attempt) {
        const uint64_t base = mix64(seed ^ mix64(i * 0x9e3779b97f4a7c15ull + attempt));
        for (int k = 0; k < 4; ++k) {
            const uint64_t v = mix64(base + 0x632be59bd9b4e019ull * (k + 1));
            w[2 * k] = (uint32_t)v;
            w[2 * k + 1] = (uint32_t)(v >> 32);
        }
        w[7] &= 0x3fffffffu;  // 254 bits
        if (Fr::is_canonical(w) || attempt > 64) break;
    }
    if (!Fr::is_canonical(w)) w[7] &= 0x0fffffffu;  // unreachable in practice; stays < r
    store_words(reinterpret_cast<uint8_t*>(out + 8 * i), w);
}

// out[i] = tau^i (canonical) for i < n, chunk consecutive powers per thread.
__global__ void k_powers(const uint32_t* __restrict__ tau_canon, uint64_t n, uint32_t chunk, uint32_t* __restrict__ out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t start = t * chunk;
    if (start >= n) return;
    uint32_t c[8];
    for (int k = 0; k < 8; ++k) c[k] = tau_canon[k];
    const Fr tau = Fr::from_canonical(c);
    Fr x = Fr::one();
    for (int bit = 63 - __clzll(start | 1); bit >= 0; --bit) {
        x = Fr::sqr(x);
        if ((start >> bit) & 1) x = Fr::mul(x, tau);
    }
    const uint64_t end = min(n, start + chunk);
    for (uint64_t i = start; i < end; ++i) {
        uint32_t o[8];
        x.to_canonical(o);
        store_words(reinterpret_cast<uint8_t*>(out + 8 * i), o);
        x = Fr::mul(x, tau);
    }
}

// a^e in Fq2 for a 256-bit exponent (8 little-endian limbs).
DV_INL Fq2 pow2(const Fq2& a, const uint32_t* e) {
    Fq2 r = Fq2::one();
    for (int i = 255; i >= 0; --i) {
        r = Fq2::sqr(r);
        if ((e[i >> 5] >> (i & 31)) & 1) r = Fq2::mul(r, a);
    }
    return r;
}

// Square root in Fq2 = Fq[u]/(u^2 + 1) for q = 3 mod 4: algorithm 9 of
// Adj and Rodriguez-Henriquez, "Square root computation over even extension
// fields" (IEEE Trans. Computers 2014).  Returns false for a non-square.
DV_INL bool sqrt2(const Fq2& a, Fq2& root) {
    uint32_t e1[8] = {FqCfg::P0, FqCfg::P1, FqCfg::P2, FqCfg::P3, FqCfg::P4, FqCfg::P5, FqCfg::P6, FqCfg::P7};
    uint32_t e2[8];
    // e1 = (q - 3) / 4, e2 = (q - 1) / 2 (q is odd and its low word exceeds 3)
    e1[0] -= 3;
    for (int i = 0; i < 8; ++i) e2[i] = e1[i];
    e2[0] += 2;
    for (int i = 0; i < 8; ++i) e2[i] = (e2[i] >> 1) | (i < 7 ? e2[i + 1] << 31 : 0u);
    for (int i = 0; i < 8; ++i) e1[i] = (e1[i] >> 2) | (i < 7 ? e1[i + 1] << 30 : 0u);
    const Fq2 a1 = pow2(a, e1);
    const Fq2 alpha = Fq2::mul(Fq2::sqr(a1), a);
    const Fq2 a0 = Fq2::mul(Fq2::conj(alpha), alpha);
    const Fq2 minus_one = Fq2::neg(Fq2::one());
    if (a0 == minus_one) return false;
    const Fq2 x0 = Fq2::mul(a1, a);
    if (alpha == minus_one) {
        root = {Fq::neg(x0.c1), x0.c0};  // u * x0
    } else {
        const Fq2 b = pow2(Fq2::add(Fq2::one(), alpha), e2);
        root = Fq2::mul(b, x0);
    }
    return Fq2::sqr(root) == a;
}

DV_INL void random_fq_words(uint64_t seed, uint64_t i, uint32_t stream, uint32_t* w) {
    for (uint32_t attempt = 0;; ++attempt) {
        const uint64_t base = mix64(seed ^ mix64(i * 0x9e3779b97f4a7c15ull + ((uint64_t)stream << 40) + attempt));
        for (int k = 0; k < 4; ++k) {
            const uint64_t v = mix64(base + 0x632be59bd9b4e019ull * (k + 1));
            w[2 * k] = (uint32_t)v;
            w[2 * k + 1] = (uint32_t)(v >> 32);
        }
        w[7] &= 0x3fffffffu;  // 254 bits
        if (Fq::is_canonical(w) || attempt > 64) break;
    }
    if (!Fq::is_canonical(w)) w[7] &= 0x0fffffffu;  // unreachable in practice; stays < q
}

// Random points of the twist curve y^2 = x^3 + 3/(9+u) over Fq2 with no
// cofactor clearing (so, with overwhelming probability, outside the order-r
// subgroup): uniform x, retried until x^3 + b' is a square.  Output: the
// 128-byte wire form x.c0 | x.c1 | y.c0 | y.c1, canonical little-endian.
__global__ void __launch_bounds__(128) k_random_twist(uint64_t seed, uint64_t n, uint8_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fq2 x, y;
    for (uint32_t attempt = 0; attempt < 256; ++attempt) {
        uint32_t w0[8], w1[8];
        random_fq_words(seed, i, 2 * attempt, w0);
        random_fq_words(seed, i, 2 * attempt + 1, w1);
        x = {Fq::from_canonical(w0), Fq::from_canonical(w1)};
        const Fq2 rhs = Fq2::add(Fq2::mul(Fq2::sqr(x), x), g2_b());
        if (sqrt2(rhs, y)) break;
    }
    uint8_t* o = out + 128 * i;
    store_canonical(o, x);
    store_canonical(o + 64, y);
}

}  // namespace

void random_twist_launch(uint64_t seed, uint64_t n, uint8_t* d_out, cudaStream_t st) {
    if (!n) return;
    k_random_twist<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(seed, n, d_out);
    DV_LAUNCH();
}

void random_fr_launch(uint64_t seed, uint64_t n, uint8_t* d_out, cudaStream_t st) {
    if (!n) return;
    k_random_fr<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(seed, n, reinterpret_cast<uint32_t*>(d_out));
    DV_LAUNCH();
}

void powers_launch(const uint8_t* d_tau, uint64_t n, uint8_t* d_out, cudaStream_t st) {
    if (!n) return;
    const uint32_t chunk = 64;
    const uint64_t threads = (n + chunk - 1) / chunk;
    k_powers<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(reinterpret_cast<const uint32_t*>(d_tau), n, chunk,
                                                                reinterpret_cast<uint32_t*>(d_out));
    DV_LAUNCH();
}

}  // namespace dv
