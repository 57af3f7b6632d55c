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

}  // namespace

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
