// Dynaverse update proofs on the device: parameters, sessions, the anchor
// proof, the fixed-anchor sparse delta proof, the verifier, and a serving
// engine that merges the pending updates of many sessions into shared
// launches.
//
// Reference (crates/protocol/src/): DynaverseParams::setup_impl
// (dynaverse.rs:104-147) over SharedSrs (srs.rs:56-197), DynamoParams
// (dynamo.rs:140-233), SliceConsistencyKey (consistency.rs:165-290) and
// KzgParams (kzg.rs:107-127); prove_anchor_traced (dynaverse.rs:149-248);
// UpdateSession::apply (dynaverse/session.rs:51-142) with its synchronous
// re-anchor (update_proof_backend, dynaverse.rs:379-470) and its sparse
// proof prove_delta_sparse_traced (dynaverse/sparse.rs:79-276); the verifier
// verify_traced in Product mode (dynaverse.rs:978-1119,
// verification.rs:37-144).  The reference composes a proof in Rust on the
// CPU and sends every MSM through OperatorBackend one synchronous call at a
// time (about 70 per sparse update); here the whole proof is composed on
// the device:
//
//  * Parameters: the trapdoor-derived base scalars are computed on the host
//    (as the reference's setup does, setup.rs:48-61), every SRS point by
//    the fixed-base kernel, and one table of c = 8 window multiples
//    (32 windows, 2 KB per base) over all G1 families (and the G2 ones), so
//    an MSM over any selection of bases adds each digit into one set of 128
//    buckets with no window combination.  Every base family a proof touches
//    lies below index 7n (witness entries below 6n, their Dynamo h images
//    below 7n), so families hold 6n, 7n or n bases.
//  * MSMs: each launch is one multi-set sequence of msm_enqueue over the
//    table, its terms given by per-term (table row, scalar index) arrays
//    expanded on the device from set descriptors (dense runs or lists), so
//    the sets of every job of a batch -- dozens of commitments per proof --
//    share one digit sort, one accumulation and one bucket reduction.
//  * Field work of a sparse update (the affected set I, |I| = a < sqrt n):
//    the vanishing polynomial A, 1/A'(x_i), the Lagrange coefficient matrix
//    of I, nine interpolations, four Cauchy sums, the local product and its
//    exact division by A -- a few batched launches over every job.  The
//    points are n-th roots of unity, so x_i - x_j = x_i (1 - w^(j-i)) and
//    1/(1 - w^d) comes from a per-parameter table: no inversion is needed.
//  * Anchor openings: the commitment of (s_t - r_t)/A (the dense quotient
//    that AnchorOpeningPolicy::Dense commits, dynaverse.rs:676-684), by an
//    exact division on a coset of the n-point domain, instead of combining
//    a cache of n single openings per wire (the Precompute policy): the
//    points are the same (dynaverse.rs:1253-1272) and no G1 transform is
//    needed at each re-anchor.  These dense sets (and a re-anchor's
//    multiplication quotient) run over a second table of the first n KZG
//    bases with c = 16 (16 windows), half the additions of the c = 8 one.
//  * Verification: every equation of the delta (and, once per anchor, of
//    the anchor) is built on the device from the proof bytes and checked by
//    the pairing kernels (pairing.cu) in one call per batch.  The
//    verifying key's G2 lines are prepared once per parameter set; the
//    G2 MSM and the lines of each proof's own G2 points run on a second
//    stream beside the dense G1 work.
//
// Proof bytes: oracle/dynaverse.py's layout, all fields in declaration
// order (G1 64 B, G2 128 B, wire format): anchor 3968 B, delta 5312 B,
// then u64 has_delta, u64 anchor_generation, u64 generation.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/dynaverse_gpu.h"
#include "backend.hpp"
#include "curve.cuh"
#include "g2.cuh"
#include "host_curve.hpp"
#include "msm.cuh"
#include "ntt.cuh"

namespace dv {

void pairing_check_device(Backend& b, const G1A* p, uint64_t terms, const G2A* q, uint64_t nq,
                          const uint32_t* d_qidx, const uint64_t* d_off, uint64_t equations, uint8_t* d_verdicts,
                          cudaStream_t st);
uint64_t pairing_prepared_bytes();
void pairing_prepare_device(const G2A* q, uint64_t nq, void* lines, uint32_t* qinf, cudaStream_t st);
void pairing_check_prepared(Backend& b, const G1A* p, uint64_t terms, const void* lines, const uint32_t* qinf,
                            const uint32_t* d_qidx, const uint64_t* d_off, uint64_t equations, uint8_t* d_verdicts,
                            cudaStream_t st);

namespace {

// ================================================================ host Fr
// Montgomery arithmetic over r on 4 x 64-bit limbs (R = 2^256), for the
// setup scalars and the session's gate checks.
namespace hf {
typedef unsigned __int128 u128;
struct Fr {
    uint64_t v[4];
};
const uint64_t P[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull, 0x30644e72e131a029ull};
const uint64_t INV = 0xc2e1f593efffffffull;  // -r^{-1} mod 2^64
const uint64_t ONE[4] = {0xac96341c4ffffffbull, 0x36fc76959f60cd29ull, 0x666ea36f7879462eull,
                         0x0e0a77c19a07df2full};
const uint64_t R2[4] = {0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull, 0x8c49833d53bb8085ull,
                        0x0216d0b17f4e44a5ull};
// ark-bn254 Fr TWO_ADIC_ROOT_OF_UNITY = 5^((r - 1) / 2^28), Montgomery form
const uint64_t TWO_ADIC[4] = {0x636e735580d13d9cull, 0xa22bf3742445ffd6ull, 0x56452ac01eb203d8ull,
                              0x1860ef942963f9e7ull};

inline bool geq(const uint64_t* a, const uint64_t* b) {
    for (int i = 3; i >= 0; --i)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}
inline void subp(uint64_t* a, const uint64_t* b) {
    uint64_t br = 0;
    for (int i = 0; i < 4; ++i) {
        u128 d = (u128)a[i] - b[i] - br;
        a[i] = (uint64_t)d;
        br = (uint64_t)(d >> 64) & 1;
    }
}
inline Fr mul(const Fr& a, const Fr& b) {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
        u128 c = 0;
        for (int j = 0; j < 4; ++j) {
            c += (u128)a.v[j] * b.v[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        const uint64_t m = t[0] * INV;
        c = ((u128)m * P[0] + t[0]) >> 64;
        for (int j = 1; j < 4; ++j) {
            c += (u128)m * P[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    Fr r = {{t[0], t[1], t[2], t[3]}};
    if (t[4] || geq(r.v, P)) subp(r.v, P);
    return r;
}
inline Fr add(const Fr& a, const Fr& b) {
    Fr r;
    uint64_t c = 0;
    for (int i = 0; i < 4; ++i) {
        u128 s = (u128)a.v[i] + b.v[i] + c;
        r.v[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    if (c || geq(r.v, P)) subp(r.v, P);
    return r;
}
inline Fr sub(const Fr& a, const Fr& b) {
    Fr r;
    uint64_t br = 0;
    for (int i = 0; i < 4; ++i) {
        u128 d = (u128)a.v[i] - b.v[i] - br;
        r.v[i] = (uint64_t)d;
        br = (uint64_t)(d >> 64) & 1;
    }
    if (br) {
        uint64_t c = 0;
        for (int i = 0; i < 4; ++i) {
            u128 s = (u128)r.v[i] + P[i] + c;
            r.v[i] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
    }
    return r;
}
inline Fr zero() { return Fr{{0, 0, 0, 0}}; }
inline Fr one() {
    Fr r;
    memcpy(r.v, ONE, 32);
    return r;
}
inline bool is_zero(const Fr& a) { return !(a.v[0] | a.v[1] | a.v[2] | a.v[3]); }
inline bool eq(const Fr& a, const Fr& b) { return !memcmp(a.v, b.v, 32); }
inline Fr from_canonical(const uint64_t* c) {
    Fr x;
    memcpy(x.v, c, 32);
    Fr r2;
    memcpy(r2.v, R2, 32);
    return mul(x, r2);
}
inline Fr from_u64(uint64_t v) {
    const uint64_t c[4] = {v, 0, 0, 0};
    return from_canonical(c);
}
inline void to_canonical(const Fr& a, uint64_t* out) {
    const Fr one_raw = {{1, 0, 0, 0}};
    const Fr c = mul(a, one_raw);
    memcpy(out, c.v, 32);
}
inline Fr pow(Fr a, const uint64_t* e, int words) {
    Fr r = one();
    for (int w = words - 1; w >= 0; --w)
        for (int bit = 63; bit >= 0; --bit) {
            r = mul(r, r);
            if ((e[w] >> bit) & 1) r = mul(r, a);
        }
    return r;
}
inline Fr pow_u64(const Fr& a, uint64_t e) { return pow(a, &e, 1); }
inline Fr inv(const Fr& a) {
    const uint64_t e[4] = {P[0] - 2, P[1], P[2], P[3]};
    return pow(a, e, 4);
}
// root of unity of order `size` (a power of two up to 2^28): TWO_ADIC squared down
inline Fr root(uint64_t size) {
    Fr w;
    memcpy(w.v, TWO_ADIC, 32);
    int log = 0;
    while ((1ull << log) < size) ++log;
    for (int i = log; i < 28; ++i) w = mul(w, w);
    return w;
}
// Montgomery's simultaneous inversion in place (every x nonzero).
inline void batch_inv(Fr* x, size_t n) {
    if (!n) return;
    std::vector<Fr> pre(n);
    Fr acc = one();
    for (size_t i = 0; i < n; ++i) {
        pre[i] = acc;
        acc = mul(acc, x[i]);
    }
    Fr t = inv(acc);
    for (size_t i = n; i-- > 0;) {
        const Fr xi = x[i];
        x[i] = mul(t, pre[i]);
        t = mul(t, xi);
    }
}
}  // namespace hf

typedef std::array<uint64_t, 4> Canon;  // canonical little-endian Fr

bool canon_ok(const uint8_t* b) {
    uint64_t w[4];
    memcpy(w, b, 32);
    return !hf::geq(w, hf::P);
}
hf::Fr mont_of(const Canon& c) { return hf::from_canonical(c.data()); }
Canon canon_of(const hf::Fr& a) {
    Canon c;
    hf::to_canonical(a, c.data());
    return c;
}

// Runs fn(lo, hi) over [0, n) on the host's cores.
void par_for(uint64_t n, const std::function<void(uint64_t, uint64_t)>& fn) {
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 4096 || hw == 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> th;
    const uint64_t chunk = (n + hw - 1) / hw;
    for (unsigned t = 0; t < hw; ++t) {
        const uint64_t lo = t * chunk, hi = std::min<uint64_t>(n, lo + chunk);
        if (lo >= hi) break;
        th.emplace_back([&fn, lo, hi] { fn(lo, hi); });
    }
    for (auto& t : th) t.join();
}

// Chunked simultaneous inversion of a long vector on the host's cores.
void par_batch_inv(std::vector<hf::Fr>& x) {
    const uint64_t n = x.size();
    const uint64_t chunk = 1 << 14;
    par_for((n + chunk - 1) / chunk, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t c = lo; c < hi; ++c) {
            const uint64_t a = c * chunk, e = std::min(n, a + chunk);
            hf::batch_inv(x.data() + a, e - a);
        }
    });
}

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// ================================================================ layout
constexpr int TC = 8, TW = 32;  // window table: c = 8, 32 windows
// The dense sets (anchor openings, a re-anchor's multiplication quotient)
// run over the first n KZG bases with wider windows: c = 16 halves their
// additions and digits against the c = 8 table at 2^15 buckets a set.
constexpr int TCD = 16, TWD = 16;
constexpr uint64_t ANCHOR_BYTES = 3968, DELTA_BYTES = 5312;
constexpr uint64_t PROOF_BYTES = DVGPU_DYNAVERSE_PROOF_BYTES;
static_assert(PROOF_BYTES == ANCHOR_BYTES + DELTA_BYTES + 24, "proof layout");

// G1 base families (rows of one SRS buffer, in this order).
enum Fam {
    F_LX, F_ALPHA, F_BETA, F_H, F_Z, F_B,  // Dynamo, 6n each (dynamo.rs:186-205)
    F_LY,                                   // 7n
    F_QAC0,                                 // six consistency qac columns, 6n each
    F_ADEG = F_QAC0 + 6,                    // 6n
    F_PQ,                                   // public quotient bases (srs.rs:84-99), 6n
    F_LAG, F_OPENU,                         // small Lagrange / single-opening bases (srs.rs:72-82), n
    F_QCD, F_QBD, F_D, F_BDEG, F_DDEG,      // common consistency columns, n
    F_KZG,                                  // [tau_x^j] G1, j < n
    F_PUBH,                                 // public-input h bases (dynamo.rs:112-124), n
    F_COUNT
};
enum Fam2 { F2_LAG, F2_KZG, F2_COUNT };

uint64_t fam_size(int f, uint64_t n) {
    if (f == F_LY) return 7 * n;
    if (f <= F_B || (f >= F_QAC0 && f <= F_PQ)) return 6 * n;
    return n;
}

// Verifying-key G2 points (Montgomery copies on the device in this order):
// the constants of the delta and anchor equations.
enum Vk2 {
    V_U, V_XM1, V_X, V_INVM, V_YM1, V_YM, V_XM, V_X2, V_G2, V_ZIN0,
    V_XMY = V_ZIN0 + 6, V_XMLY, V_PZD, V_MD, V_COUNT
};

// Proof slot offsets (bytes).  Anchor (dynaverse AnchorProof fields):
constexpr uint64_t A_WIRES = 0, A_S5G2 = 384, A_W = 512, A_H = 576, A_DYN = 640, A_CONS = 1152, A_PZQ = 3840,
                   A_MQ = 3904;
// Delta (DeltaProof fields), relative to the delta part:
constexpr uint64_t D_WIRES = 0, D_W = 384, D_H = 448, D_DYN = 512, D_CONS = 1024, D_PZQ = 3712, D_AFF1 = 3776,
                   D_AFF2 = 3840, D_UNAFF1 = 3968, D_UNAFF2 = 4032, D_ALOC = 4160, D_CLOC = 4352, D_US5 = 4544,
                   D_AOPEN = 4672, D_COPEN = 4864, D_UZERO = 5056, D_LQ = 5248;
// Dynamo field order inside a proof: alpha, beta, h, z, b, q, instance_z,
// instance_h (64 B each); consistency: six slices of qac, qcd, qbd, d,
// a_degree, b_degree, d_degree (448 B each).
constexpr int DY_IZ = 6, DY_IH = 7;

// Per-job record in the output arena: delta fields (5312 B; for a re-anchor
// the delta's linear fields), side slots ([public]_h before the update, the
// MSM of the public differences -- or of all public inputs for a fresh
// anchor --, [public]_h after), then anchor fields (3968 B).
constexpr uint64_t SIDE_PUB = 5312, SIDE_PDIFF = 5312 + 64, SIDE_PUBNEW = 5312 + 128, REC_ANCHOR = 5504;
constexpr uint64_t JOB_BYTES = REC_ANCHOR + 3968;
static_assert(REC_ANCHOR % 128 == 0 && JOB_BYTES % 128 == 0, "record alignment");

// ================================================================ device kernels
// Canonical words <-> Montgomery.
DV_INL Fr mont(const Fr& canonical) { return Fr::from_canonical(canonical.v); }
DV_INL Fr canon(const Fr& m) {
    Fr c;
    m.to_canonical(c.v);
    return c;
}
// Canonical affine G1 bytes (all zero = infinity) -> Montgomery affine.
DV_INL G1A load_g1(const uint8_t* p) {
    uint32_t x[8], y[8];
    load_words(p, x);
    load_words(p + 32, y);
    return {Fq::from_canonical(x), Fq::from_canonical(y)};
}
DV_INL void store_g1(uint8_t* p, const G1A& a) {
    store_canonical(p, a.x);
    store_canonical(p + 32, a.y);
}
DV_INL G2A load_g2(const uint8_t* p) {
    uint32_t w[8];
    G2A r;
    load_words(p, w);
    r.x.c0 = Fq::from_canonical(w);
    load_words(p + 32, w);
    r.x.c1 = Fq::from_canonical(w);
    load_words(p + 64, w);
    r.y.c0 = Fq::from_canonical(w);
    load_words(p + 96, w);
    r.y.c1 = Fq::from_canonical(w);
    return r;
}

// A segment of an MSM set (a set is one or more consecutive segments):
// `count` terms, point rows and scalar indices
//   kind 0 (dense run):  row0 + j,                 sc0 + j
//   kind 1 (list):       row0 + lrow[list + j],    lsc[list + j]
//   kind 2 (list rows):  row0 + lrow[list + j],    sc0 + j
struct SetDesc {
    uint32_t kind, count, row0, sc0, list, pad;
};

// term_off: first term of each segment (segments + 1 entries).
__global__ void k_dv_expand(uint32_t total, uint32_t sets, const uint32_t* __restrict__ term_off,
                            const SetDesc* __restrict__ d, const uint32_t* __restrict__ lrow,
                            const uint32_t* __restrict__ lsc, uint32_t* __restrict__ tpoint,
                            uint32_t* __restrict__ tscalar) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    uint32_t lo = 0, hi = sets;  // the set s with term_off[s] <= i < term_off[s + 1]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (term_off[mid] <= i) lo = mid; else hi = mid;
    }
    const SetDesc s = d[lo];
    const uint32_t j = i - term_off[lo];
    if (s.kind == 0) {
        tpoint[i] = s.row0 + j;
        tscalar[i] = s.sc0 + j;
    } else {
        tpoint[i] = s.row0 + lrow[s.list + j];
        tscalar[i] = s.kind == 1 ? lsc[s.list + j] : s.sc0 + j;
    }
}

// Set sums -> canonical affine bytes at out + off[k] (~0: not written).
template <class F>
__global__ void k_dv_affine(const XYZZ<F>* __restrict__ sums, uint32_t count, const uint64_t* __restrict__ off,
                            uint8_t* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count || off[k] == ~0ull) return;
    const Affine<F> a = sums[k].to_affine();
    store_canonical(out + off[k], a.x);
    store_canonical(out + off[k] + sizeof(F), a.y);
}

// Byte copies inside the output arena (duplicate proof fields and
// constants): dst, src, bytes (multiples of 16).
struct CopyDesc {
    uint8_t* dst;
    const uint8_t* src;
    uint64_t bytes;
};
__global__ void k_dv_copy(uint32_t count, const CopyDesc* __restrict__ c) {
    const uint32_t k = blockIdx.y;
    if (k >= count) return;
    const CopyDesc d = c[k];
    for (uint64_t b = 16ull * (blockIdx.x * blockDim.x + threadIdx.x); b < d.bytes; b += 16ull * gridDim.x * blockDim.x)
        *reinterpret_cast<uint4*>(d.dst + b) = *reinterpret_cast<const uint4*>(d.src + b);
}

// ---------------------------------------------------------------- anchor witness helpers
// h_j = w_j - w_sigma(j) for j < 7n (w is zero from 6n on; sigma swaps
// i <-> 6n+i and 2n+i <-> 3n+i, toy_circuit.rs:17-27): derive_h_sparse of a
// dense witness (dynamo.rs:462-476).
__global__ void k_dv_h(const Fr* __restrict__ w, uint32_t n, Fr* __restrict__ h) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 7 * n) return;
    uint32_t s = j;
    if (j < n) s = 6 * n + j;
    else if (j >= 6 * n) s = j - 6 * n;
    else if (j >= 2 * n && j < 3 * n) s = j + n;
    else if (j >= 3 * n && j < 4 * n) s = j - n;
    const Fr a = j < 6 * n ? w[j] : Fr::zero();
    const Fr b = s < 6 * n ? w[s] : Fr::zero();
    h[j] = Fr::sub(a, b);  // canonical operands: canonical difference
}

// dst[i] = i < len ? src[i] : 0 for i < size.
__global__ void k_dv_pad(const Fr* __restrict__ src, uint64_t len, Fr* __restrict__ dst, uint64_t size) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < size) dst[i] = i < len ? src[i] : Fr::zero();
}
// a[i] = a[i] b[i] (canonical in and out).
__global__ void k_dv_pmul(Fr* __restrict__ a, const Fr* __restrict__ b, uint64_t size) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < size) a[i] = Fr::mul(a[i], mont(b[i]));
}
// Multiplication quotient (s4 s5 - s6) / (X^n - 1) of the anchor
// (dynaverse.rs:224-229, divide_exact_by_xn_minus_one): with P = s4 s5
// (2n coefficients, the last zero) and N = P - s6, the quotient is
// q_k = P_(n+k) (k < n - 1) and the division is exact iff N_k + P_(n+k) = 0
// for every k < n.
__global__ void k_dv_mq(const Fr* __restrict__ p, const Fr* __restrict__ s6, uint32_t n, Fr* __restrict__ q,
                        uint32_t* __restrict__ status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const Fr hi = p[n + k];
    if (!Fr::add(Fr::sub(p[k], s6[k]), hi).is_zero()) atomicOr(status, 4u);
    if (k + 1 < n) q[k] = hi;
}

// ---------------------------------------------------------------- sparse update: field work
// One job = one sparse update over an affected set of a points
// x_k = w^e_k of the n-point domain.  Offsets are in Fr elements of the
// scalar arena (canonical) and of the scratch (Montgomery).
struct FieldJob {
    uint32_t a, aff;     // affected count; offset of e_k in the list array
    uint32_t in, out;    // arena: 6a inputs (anchor values, delta values of wires 3..5); 19a + 1 outputs
    uint32_t scr, mat;   // scratch: 22a + 1; Lagrange matrix a * a
    uint32_t dense;      // arena: 4 rows of n (anchor-opening numerators, A)
    uint32_t status;     // index of the job's status word
    const Fr* coef;      // the session's anchor coefficients s4 | s5 | s6 (canonical, 3n)
};
// output offsets within a job's 19a + 1 outputs
DV_INL uint32_t o_A(uint32_t) { return 0; }
DV_INL uint32_t o_B(uint32_t a) { return a + 1; }
DV_INL uint32_t o_R(uint32_t a, int t) { return 2 * a + 1 + t * a; }
DV_INL uint32_t o_RS(uint32_t a, int t) { return 5 * a + 1 + t * a; }
DV_INL uint32_t o_ZQ(uint32_t a, int t) { return 8 * a + 1 + t * a; }
DV_INL uint32_t o_LAG(uint32_t a, int t) { return 11 * a + 1 + t * a; }
DV_INL uint32_t o_OPN(uint32_t a, int t) { return 14 * a + 1 + t * a; }
DV_INL uint32_t o_U1(uint32_t a) { return 17 * a + 1; }
DV_INL uint32_t o_LQ(uint32_t a) { return 18 * a + 1; }
// scratch offsets
DV_INL uint32_t s_X(uint32_t) { return 0; }
DV_INL uint32_t s_XI(uint32_t a) { return a; }
DV_INL uint32_t s_W(uint32_t a) { return 2 * a; }
DV_INL uint32_t s_D(uint32_t a) { return 3 * a; }
DV_INL uint32_t s_CW(uint32_t a) { return 4 * a; }
DV_INL uint32_t s_CV(uint32_t a, int t) { return 5 * a + t * a; }
DV_INL uint32_t s_AM(uint32_t a) { return 8 * a; }
DV_INL uint32_t s_V(uint32_t a, int row) { return 9 * a + 1 + row * a; }

struct FieldCtx {
    const FieldJob* jobs;
    const uint32_t* kjob;  // prefix sums of a over jobs (jobs + 1 entries)
    uint32_t njobs;
    const uint32_t* list;  // affected indices e_k
    const Fr* wpow;        // w^k, k < n (Montgomery)
    const Fr* inv1m;       // 1 / (1 - w^k), 0 < k < n (Montgomery)
    uint32_t n;
    Fr n_m, ninv_m;        // n and 1/n (Montgomery)
    Fr* arena;             // canonical
    Fr* scr;               // Montgomery
    uint32_t* status;
};

DV_INL uint32_t job_of(const uint32_t* pre, uint32_t njobs, uint32_t i) {
    uint32_t lo = 0, hi = njobs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pre[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Per point: x_k, 1/x_k, w_k = 1/A'(x_k) and A'(x_k), with
// A'(x_k) = x_k^(a-1) prod_{j != k} (1 - w^(e_j - e_k)) and
// 1/A'(x_k) = x_k^-(a-1) prod_{j != k} 1/(1 - w^(e_j - e_k)); the B scalars
// n w_k / x_k (Z'(x_k)/A'(x_k), sparse.rs:131-134) and the Montgomery rows
// the interpolations and Cauchy sums read.
// An element of Fr from lane (this lane xor m) of the warp.
DV_INL Fr shfl_xor_fr(const Fr& a, int m) {
    Fr r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_xor_sync(0xffffffffu, a.v[i], m);
    return r;
}

DV_INL Fr shfl_up_fr(const Fr& a, int d) {
    Fr r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_up_sync(0xffffffffu, a.v[i], d);
    return r;
}

// One warp per affected point k: the products over j != k are split over
// the lanes and combined by a butterfly, so the chain is a / 32 + 5 products
// long instead of a.
__global__ void k_dv_geom(FieldCtx c) {
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= c.kjob[c.njobs]) return;  // uniform across the warp
    const uint32_t jb = job_of(c.kjob, c.njobs, gw);
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a, k = gw - c.kjob[jb], mask = c.n - 1;
    const uint32_t* e = c.list + J.aff;
    const uint32_t ek = e[k];
    const Fr one = Fr::one();
    Fr pinv = one, pd = one;
    for (uint32_t j = lane; j < a; j += 32) {
        if (j == k) continue;
        const uint32_t d = (e[j] - ek) & mask;
        const auto pr = Fr::mul2(pinv, c.inv1m[d], pd, Fr::sub(one, c.wpow[d]));
        pinv = pr.r0;
        pd = pr.r1;
    }
    for (int m = 16; m >= 1; m >>= 1) {
        const Fr oi = shfl_xor_fr(pinv, m), od = shfl_xor_fr(pd, m);
        const auto pr = Fr::mul2(pinv, oi, pd, od);
        pinv = pr.r0;
        pd = pr.r1;
    }
    if (lane) return;
    const Fr x = c.wpow[ek], xi = c.wpow[(c.n - ek) & mask];
    {
        const auto pr = Fr::mul2(pinv, c.wpow[(uint32_t)(((uint64_t)((c.n - ek) & mask) * (a - 1)) & mask)], pd,
                                 c.wpow[(uint32_t)(((uint64_t)ek * (a - 1)) & mask)]);
        pinv = pr.r0;
        pd = pr.r1;
    }
    Fr* s = c.scr + J.scr;
    s[s_X(a) + k] = x;
    s[s_XI(a) + k] = xi;
    s[s_W(a) + k] = pinv;
    s[s_D(a) + k] = pd;
    c.arena[J.out + o_B(a) + k] = canon(Fr::mul(Fr::mul(c.n_m, xi), pinv));
    const Fr* in = c.arena + J.in;
    for (int t = 0; t < 3; ++t) {
        const Fr al = mont(in[t * a + k]);
        const Fr v = mont(in[(3 + t) * a + k]);
        s[s_V(a, t) + k] = al;
        s[s_V(a, 3 + t) + k] = v;
        // zero-quotient values v / w_k * x_k / n (sparse.rs:222)
        s[s_V(a, 6 + t) + k] = Fr::mul(Fr::mul(v, pd), Fr::mul(x, c.ninv_m));
        s[s_V(a, 10 + t) + k] = Fr::mul(v, x);  // Cauchy weights v x (sparse.rs:208)
    }
    s[s_V(a, 9) + k] = pinv;  // Cauchy weights of the tree's own weights (sparse.rs:176)
}

// A = prod (X - x_k), one block per job: A at the N-th roots of unity
// (N = the power of two above a; a sparse job has a < sqrt(n), so N <= n and
// the points come from the table of w^k), one warp per point with the
// product split over its lanes, then an inverse transform of size N in
// shared memory.  The chain is about a / 32 + log N + 5 products, against a
// for the product taken one factor at a time.
__global__ void __launch_bounds__(1024) k_dv_vanish(FieldCtx c) {
    extern __shared__ Fr sm[];
    const uint32_t jb = blockIdx.x;
    if (jb >= c.njobs) return;
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a;
    Fr* s = c.scr + J.scr;
    uint32_t logN = 0;
    while ((1u << logN) < a + 1) ++logN;
    const uint32_t N = 1u << logN, step = c.n >> logN, mask = c.n - 1;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    for (uint32_t i = warp; i < N; i += nwarp) {
        const Fr y = c.wpow[(i * step) & mask];
        Fr p = Fr::one();
        for (uint32_t k = lane; k < a; k += 32) p = Fr::mul(p, Fr::sub(y, s[s_X(a) + k]));
        for (int m = 16; m >= 1; m >>= 1) p = Fr::mul(p, shfl_xor_fr(p, m));
        if (lane == 0) sm[logN ? __brev(i) >> (32 - logN) : 0] = p;
    }
    __syncthreads();
    // inverse transform (decimation in time, bit-reversed input)
    for (uint32_t half = 1; half < N; half <<= 1) {
        const uint32_t stride = c.n / (2 * half);
        for (uint32_t b = threadIdx.x; b < N / 2; b += blockDim.x) {
            const uint32_t j = b % half, i0 = (b / half) * 2 * half + j, i1 = i0 + half;
            const Fr tw = c.wpow[(c.n - j * stride) & mask];  // w_(2 half)^(-j)
            const Fr u = sm[i0], t = Fr::mul(sm[i1], tw);
            sm[i0] = Fr::add(u, t);
            sm[i1] = Fr::sub(u, t);
        }
        __syncthreads();
    }
    Fr sc;  // 1 / N = (n / N) / n
    for (int i = 0; i < 8; ++i) sc.v[i] = i ? 0u : step;
    const Fr ninv = Fr::mul(c.ninv_m, mont(sc));
    for (uint32_t j = threadIdx.x; j <= a; j += blockDim.x) {
        const Fr v = Fr::mul(sm[j], ninv);
        s[s_AM(a) + j] = v;
        c.arena[J.out + o_A(a) + j] = canon(v);
    }
}

// Lagrange coefficient matrix of the affected set:
// M[k][j] = w_k q_(k,j), q_k = A / (X - x_k) by synthetic division:
// q_(a-1) = A_a, q_(t-1) = A_t + x q_t.  One warp per k: lane l runs the
// steps of one chunk of t, whose effect is the affine map
// q -> x^len q + C_l; a warp scan of those maps gives every lane the value
// entering its chunk, so the chain is about a / 16 + 10 products long.
__global__ void k_dv_lagmat(FieldCtx c) {
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= c.kjob[c.njobs]) return;  // uniform across the warp
    const uint32_t jb = job_of(c.kjob, c.njobs, gw);
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a, k = gw - c.kjob[jb];
    const Fr* s = c.scr + J.scr;
    const Fr* am = s + s_AM(a);
    Fr* m = c.scr + J.mat + (uint64_t)k * a;
    const Fr x = s[s_X(a) + k], w = s[s_W(a) + k];
    // lane l: t from hi down to lo (lane 0 holds the top), steps t = hi .. lo
    const int L = (int)((a + 31) / 32);
    const int hi = (int)a - 1 - (int)lane * L, lo = hi - L + 1 < 0 ? 0 : hi - L + 1;
    const bool live = hi >= 0;
    Fr alpha = Fr::one(), cst = Fr::zero();
    if (live)
        for (int t = hi; t >= lo; --t) {
            const auto pr = Fr::mul2(alpha, x, cst, x);
            alpha = pr.r0;
            cst = Fr::add(am[t], pr.r1);
        }
    // inclusive scan of the maps in lane order: (alpha, cst) after the earlier lanes' maps
    for (int d = 1; d < 32; d <<= 1) {
        const Fr pa = shfl_up_fr(alpha, d), pc = shfl_up_fr(cst, d);
        if ((int)lane >= d) {
            const auto pr = Fr::mul2(alpha, pa, alpha, pc);
            alpha = pr.r0;
            cst = Fr::add(pr.r1, cst);
        }
    }
    // the value entering this lane's chunk: the earlier lanes' composition applied to A_a
    const Fr ea = shfl_up_fr(alpha, 1), ec = shfl_up_fr(cst, 1);
    const Fr top = am[a];
    Fr q = lane == 0 ? top : Fr::add(Fr::mul(ea, top), ec);
    if (!live) return;
    m[hi] = Fr::mul(w, q);
    for (int t = hi; t > lo; --t) {
        q = Fr::add(am[t], Fr::mul(x, q));
        m[t - 1] = Fr::mul(w, q);
    }
}

// Rows 0..8: interpolation coefficients f_j = sum_k M[k][j] v_k of the
// anchor values, delta values and zero-quotient values of wires 4..6;
// rows 9..12: Cauchy sums sum_(j != k) u_j / (x_k - x_j)
// = (1/x_k) sum_(j != k) u_j / (1 - w^(e_j - e_k)) (SubproductTree::
// cauchy_sums, domain/fast.rs:118-139) of the weights and of v x.
__global__ void k_dv_rows(FieldCtx c) {
    // one warp per (affected point, row); the lanes split the sum
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= 13 * c.kjob[c.njobs]) return;  // uniform across the warp
    const uint32_t row_job = gw / 13;  // flattened (job, idx) with 13 rows each
    const uint32_t row = gw % 13;
    const uint32_t jb = job_of(c.kjob, c.njobs, row_job);
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a, idx = row_job - c.kjob[jb], mask = c.n - 1;
    const Fr* s = c.scr + J.scr;
    const Fr* v = s + s_V(a, row);
    Fr acc = Fr::zero();
    if (row < 9) {
        const Fr* m = c.scr + J.mat + idx;
        for (uint32_t k = lane; k < a; k += 32) acc = Fr::add(acc, Fr::mul(m[(uint64_t)k * a], v[k]));
    } else {
        const uint32_t* e = c.list + J.aff;
        const uint32_t ek = e[idx];
        for (uint32_t j = lane; j < a; j += 32) {
            if (j == idx) continue;
            acc = Fr::add(acc, Fr::mul(v[j], c.inv1m[(e[j] - ek) & mask]));
        }
    }
    for (int m = 16; m >= 1; m >>= 1) acc = Fr::add(acc, shfl_xor_fr(acc, m));
    if (lane) return;
    if (row < 9) {
        const uint32_t o = row < 3 ? o_R(a, row) : row < 6 ? o_RS(a, row - 3) : o_ZQ(a, row - 6);
        c.arena[J.out + o + idx] = canon(acc);
    } else {
        acc = Fr::mul(acc, s[s_XI(a) + idx]);
        Fr* dst = c.scr + J.scr + (row == 9 ? s_CW(a) : s_CV(a, row - 10));
        dst[idx] = acc;
    }
}

// Lagrange / opening scalars of the changed openings (sparse.rs:210-219):
// v_k cw_k + w_k cv_k / x_k and v_k w_k.
__global__ void k_dv_combine(FieldCtx c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.kjob[c.njobs]) return;
    const uint32_t jb = job_of(c.kjob, c.njobs, i);
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a, k = i - c.kjob[jb];
    const Fr* s = c.scr + J.scr;
    const Fr w = s[s_W(a) + k], cw = s[s_CW(a) + k], wx = Fr::mul(w, s[s_XI(a) + k]);
    for (int t = 0; t < 3; ++t) {
        const Fr v = s[s_V(a, 3 + t) + k];
        const Fr lag = Fr::add(Fr::mul(v, cw), Fr::mul(wx, s[s_CV(a, t) + k]));
        c.arena[J.out + o_LAG(a, t) + k] = canon(lag);
        c.arena[J.out + o_OPN(a, t) + k] = canon(Fr::mul(v, w));
    }
}

// updated_t = r_t + r*_t; the local product u0 u1 - u2 divided by the monic
// A (sparse.rs:225-236), quotient and remainder check, one block per job.
// Shared memory: u0 (canonical), u1 (Montgomery), N (2a - 1, canonical).
__global__ void k_dv_quot(FieldCtx c) {
    extern __shared__ Fr sm[];
    const uint32_t jb = blockIdx.x;
    if (jb >= c.njobs) return;
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a;
    if (!a) return;
    Fr* u0 = sm;
    Fr* u1m = sm + a;
    Fr* N = sm + 2 * a;
    Fr* out = c.arena + J.out;
    const Fr* am = c.scr + J.scr + s_AM(a);
    for (uint32_t j = threadIdx.x; j < a; j += blockDim.x) {
        u0[j] = Fr::add(out[o_R(a, 0) + j], out[o_RS(a, 0) + j]);
        const Fr u1 = Fr::add(out[o_R(a, 1) + j], out[o_RS(a, 1) + j]);
        out[o_U1(a) + j] = u1;
        u1m[j] = mont(u1);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < 2 * a - 1; k += blockDim.x) {
        Fr acc = Fr::zero();
        const uint32_t lo = k >= a ? k - a + 1 : 0, hi = k < a ? k : a - 1;
        for (uint32_t j = lo; j <= hi; ++j) acc = Fr::add(acc, Fr::mul(u0[j], u1m[k - j]));
        if (k < a) acc = Fr::sub(acc, Fr::add(out[o_R(a, 2) + k], out[o_RS(a, 2) + k]));
        N[k] = acc;
    }
    __syncthreads();
    // long division by the monic A of degree a: N has degree <= 2a - 2
    for (int i = (int)a - 2; i >= 0; --i) {
        const Fr q = N[i + a];
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < a; j += blockDim.x) N[i + j] = Fr::sub(N[i + j], Fr::mul(q, am[j]));
        if (threadIdx.x == 0) out[o_LQ(a) + i] = q;
        __syncthreads();
    }
    for (uint32_t j = threadIdx.x; j < a; j += blockDim.x)
        if (!N[j].is_zero()) atomicOr(c.status + J.status, 1u);
}

// Anchor openings (s_t - r_t) / A: numerators and A, four rows of n each.
__global__ void k_dv_numer(FieldCtx c) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t per = 4ull * c.n;
    if (i >= per * c.njobs) return;
    const uint32_t jb = (uint32_t)(i / per);
    const FieldJob J = c.jobs[jb];
    const uint32_t a = J.a;
    if (!a) return;
    const uint32_t r = (uint32_t)((i % per) / c.n), k = (uint32_t)(i % c.n);
    Fr v;
    if (r < 3) {
        v = J.coef[(uint64_t)r * c.n + k];
        if (k < a) v = Fr::sub(v, c.arena[J.out + o_R(a, r) + k]);
    } else {
        v = k <= a ? c.arena[J.out + o_A(a) + k] : Fr::zero();
    }
    c.arena[J.dense + (uint64_t)r * c.n + k] = v;
}

// Coset values of the numerators divided by those of A (5 H meets no root
// of A: its roots are n-th roots of unity).
// One thread per DQ consecutive coset points (8: a longer chain costs more
// latency in a lone update than it saves in a batch): their A values inverted
// together by Montgomery's trick (one inversion, 3 (DQ - 1) products).  A has
// its roots in H, so no value on the coset 5 H is zero.
constexpr uint32_t DQ = 8;
__global__ void k_dv_divq(FieldCtx c) {
    const uint32_t chunks = (c.n + DQ - 1) / DQ;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)chunks * c.njobs) return;
    const uint32_t jb = (uint32_t)(i / chunks), k0 = (uint32_t)(i % chunks) * DQ;
    const FieldJob J = c.jobs[jb];
    if (!J.a) return;
    Fr* rows = c.arena + J.dense;
    const Fr* av = rows + 3ull * c.n + k0;
    const uint32_t m = min(DQ, c.n - k0);
    Fr pre[DQ];  // pre[j] = a_0 ... a_(j-1) (Montgomery)
    Fr acc = Fr::one();
    for (uint32_t j = 0; j < m; ++j) {
        pre[j] = acc;
        acc = Fr::mul(acc, mont(av[j]));
    }
    Fr inv = Fr::inv(acc);  // 1 / (a_0 ... a_(m-1))
    for (int j = (int)m - 1; j >= 0; --j) {
        const Fr a = mont(av[j]);
        const Fr ainv = Fr::mul(inv, pre[j]);
        inv = Fr::mul(inv, a);
        for (int t = 0; t < 3; ++t) rows[(uint64_t)t * c.n + k0 + j] = Fr::mul(rows[(uint64_t)t * c.n + k0 + j], ainv);
    }
}

// An exact quotient has degree < n - a.
__global__ void k_dv_degcheck(FieldCtx c) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3ull * c.n * c.njobs) return;
    const uint32_t jb = (uint32_t)(i / (3ull * c.n));
    const FieldJob J = c.jobs[jb];
    const uint64_t rk = i % (3ull * c.n);
    const uint32_t k = (uint32_t)(rk % c.n);
    if (!J.a || k < c.n - J.a) return;
    if (!c.arena[J.dense + rk].is_zero()) atomicOr(c.status + J.status, 2u);
}

// ---------------------------------------------------------------- verification
// The pairing-product equations of verify_traced (dynaverse.rs:1018-1119;
// dynamo_verify_with_checks, dynamo.rs:326-342; verify_six_with_checks /
// verify_with_checks, consistency.rs:49-114), one warp per proof, right-
// hand sides negated as product_equal does (verification.rs:80-92).  G2
// terms index the batch's G2 array: the verifying-key constants (Vk2), then
// each proof's own G2 points.
struct VerifyJob {
    uint8_t* rec;           // the job's record in the output arena
    const uint8_t* anchor;  // anchor proof bytes (== rec for an anchor job)
    uint32_t kind;          // 0 anchor, 1 delta, 2 anchor of a proof with a delta
    uint32_t term, fresh;   // first term; first own G2 point (index into q)
    uint32_t status;
};
constexpr uint32_t ANCHOR_TERMS = 84, ANCHOR_EQS = 37, DELTA_TERMS = 108, DELTA_EQS = 49;

struct Emit {
    G1A* p;
    uint32_t* q;
    uint32_t k;
    DV_INL void t(const G1A& g, uint32_t qi) {
        p[k] = g;
        q[k] = qi;
        ++k;
    }
};
DV_INL G1A g1_sub(const G1A& a, const G1A& b) { return G1X::add_affine(G1X::from_affine(a), b.neg()).to_affine(); }
DV_INL G1A g1_add(const G1A& a, const G1A& b) { return G1X::add_affine(G1X::from_affine(a), b).to_affine(); }

// ---------------------------------------------------------------- incremental re-anchor
// Every anchor field but the multiplication quotient is a commitment linear
// in the witness (prove_anchor_traced, dynaverse.rs:149-248): for the new
// anchor w' = w + delta it is the old field plus the same commitment of the
// delta, which the sparse pipeline computes anyway (the reference's
// FixedLinear, dynaverse/sparse_linear.rs:495-559, adds them the same way).
// Field f of a re-anchor: (anchor offset, offset of the delta's field).
DV_INL void rebase_field(uint32_t f, uint64_t& ao, uint64_t& dof) {
    if (f < 6) { ao = A_WIRES + 64 * f; dof = D_WIRES + 64 * f; }
    else if (f == 6) { ao = A_W; dof = D_DYN + 64 * 6; }
    else if (f == 7) { ao = A_H; dof = D_DYN + 64 * 7; }
    else if (f < 16) { ao = A_DYN + 64 * (f - 8); dof = D_DYN + 64 * (f - 8); }
    else if (f < 58) { ao = A_CONS + 64 * (f - 16); dof = D_CONS + 64 * (f - 16); }
    else if (f == 58) { ao = A_PZQ; dof = D_PZQ; }
    else { ao = A_S5G2; dof = D_AFF2; }  // G2: s5 over the delta of wire s5
}
constexpr uint32_t REBASE_FIELDS = 60;
struct RebaseJob {
    uint8_t* rec;       // the job's record: delta fields, then the new anchor at REC_ANCHOR
    const uint8_t* old; // the current anchor proof bytes
};
// Fields [f0, f1) of every job (the G1 fields and the G2 field run on
// different streams, each after the MSM that produces its delta).
__global__ void k_dv_rebase(const RebaseJob* __restrict__ jobs, uint32_t njobs, uint32_t f0, uint32_t f1) {
    const uint32_t w = f1 - f0;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= njobs * w) return;
    const RebaseJob J = jobs[i / w];
    const uint32_t f = f0 + i % w;
    uint64_t ao, dof;
    rebase_field(f, ao, dof);
    uint8_t* out = J.rec + REC_ANCHOR + ao;
    if (f + 1 < REBASE_FIELDS) {
        store_g1(out, g1_add(load_g1(J.old + ao), load_g1(J.rec + dof)));
    } else {
        const G2A r = G2X::add_affine(G2X::from_affine(load_g2(J.old + ao)), load_g2(J.rec + dof)).to_affine();
        store_canonical(out, r.x);
        store_canonical(out + 64, r.y);
    }
}
// arena[dst[k]] = arena[src[k]]
__global__ void k_dv_scatter(const uint32_t* __restrict__ pairs, uint32_t count, Fr* __restrict__ arena) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) arena[pairs[2 * k]] = arena[pairs[2 * k + 1]];
}
// out = x + y (canonical)
__global__ void k_dv_vadd(Fr* __restrict__ out, const Fr* __restrict__ x, const Fr* __restrict__ y, uint64_t count) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] = Fr::add(x[k], y[k]);
}

// Dynamo fields at p (alpha, beta, h, z, b, q, instance_z, instance_h).
DV_INL void emit_dynamo(Emit& e, const uint8_t* p) {
    const G1A alpha = load_g1(p), beta = load_g1(p + 64), h = load_g1(p + 128), z = load_g1(p + 192),
              b = load_g1(p + 256), q = load_g1(p + 320), iz = load_g1(p + 384), ih = load_g1(p + 448);
    e.t(iz, V_U); e.t(alpha.neg(), V_XM1); e.t(beta.neg(), V_X); e.t(ih.neg(), V_INVM); e.t(q.neg(), V_YM1);
    e.t(iz, V_YM); e.t(z.neg(), V_G2);
    e.t(ih, V_XM); e.t(h.neg(), V_G2);
    e.t(beta, V_X2); e.t(b.neg(), V_G2);
}
// Consistency slice t: a = the big-domain commitment, wires at w, fields at c.
DV_INL void emit_slice(Emit& e, const G1A& a, const uint8_t* w, const uint8_t* c, int t) {
    const uint8_t* s = c + 448 * t;
    const G1A b = load_g1(w + 64 * t);
    const G1A qac = load_g1(s), qcd = load_g1(s + 64), qbd = load_g1(s + 128), d = load_g1(s + 192),
              adeg = load_g1(s + 256), bdeg = load_g1(s + 320), ddeg = load_g1(s + 384);
    e.t(g1_sub(a, d), V_G2); e.t(qac.neg(), V_ZIN0 + t); e.t(qcd.neg(), V_XMY);
    e.t(g1_sub(b, d), V_G2); e.t(qbd.neg(), V_XMLY);
    e.t(a, V_YM); e.t(adeg.neg(), V_G2);
    e.t(b, V_YM); e.t(bdeg.neg(), V_G2);
    e.t(d, V_XM); e.t(ddeg.neg(), V_G2);
}
constexpr uint32_t DYNAMO_TERMS = 11, SLICE_TERMS = 11, TAIL_TERMS = DYNAMO_TERMS + 6 * SLICE_TERMS;

// Each job's own G2 points into q (the batch's G2 array, after the
// verifying key): an anchor's s5 commitment; a delta's affected, unaffected
// and updated-s5 commitments.  One thread per job.
__global__ void k_dv_fresh(const VerifyJob* __restrict__ jobs, uint32_t njobs, G2A* __restrict__ q) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const VerifyJob J = jobs[j];
    G2A* o = q + V_COUNT + J.fresh;
    if (J.kind != 1) {
        o[0] = load_g2(J.anchor + A_S5G2);
    } else {
        o[0] = load_g2(J.rec + D_AFF2);
        o[1] = load_g2(J.rec + D_UNAFF2);
        o[2] = load_g2(J.rec + D_US5);
    }
}

// One 32-thread block per (proof, piece), its first lane working: pieces in
// different blocks do not serialise on divergent branches, and a block of
// one warp leaves the register budget to the field arithmetic.  Every term has a
// fixed position, so the pieces write independently: piece 0 the dynamo
// terms, 1..6 the six consistency slices, then the tail (the public-zero,
// multiplication and, for a delta, the affected-set and opening equations)
// over pieces 7..13, and the group identities and the new [public]_h on
// piece 14.  Each affine normalisation takes a field inversion, so spreading
// them over the pieces shortens the chain to two inversions.
constexpr uint32_t TERM_PIECES = 15;
__global__ void k_dv_terms(const VerifyJob* __restrict__ jobs, uint32_t njobs, G1A g1, G1A mvg1,
                           G1A* __restrict__ p, uint32_t* __restrict__ qidx, uint32_t* __restrict__ status) {
    if (blockIdx.x >= njobs || threadIdx.x) return;
    const uint32_t lane = blockIdx.y;  // the piece
    const VerifyJob J = jobs[blockIdx.x];
    const uint8_t* A = J.anchor;
    uint8_t* r = J.rec;
    const bool delta = J.kind == 1;
    const uint8_t* dyn = delta ? r + D_DYN : A + A_DYN;
    const uint8_t* wires = delta ? r + D_WIRES : A + A_WIRES;
    auto at = [&](uint32_t k) { return Emit{p + J.term, qidx + J.term, k}; };
    if (lane == 0) {
        Emit e = at(0);
        emit_dynamo(e, dyn);
        return;
    }
    if (lane <= 6) {
        Emit e = at(DYNAMO_TERMS + SLICE_TERMS * (lane - 1));
        emit_slice(e, load_g1(delta ? r + D_W : A + A_W), wires, delta ? r + D_CONS : A + A_CONS, (int)lane - 1);
        return;
    }
    bool ok = true;
    if (!delta) {
        const uint32_t s5 = V_COUNT + J.fresh;
        if (lane == 7) {
            const G1A w = load_g1(A + A_W);
            const G1A w3 = load_g1(A + A_WIRES + 192), w4 = load_g1(A + A_WIRES + 256), w5 = load_g1(A + A_WIRES + 320);
            Emit e = at(TAIL_TERMS);
            e.t(load_g1(A + A_PZQ), V_PZD); e.t(w.neg(), V_G2);
            e.t(w4, V_G2); e.t(g1.neg(), s5);
            e.t(w3, s5); e.t(w5.neg(), V_G2); e.t(load_g1(A + A_MQ).neg(), V_MD);
        } else if (lane == 8) {
            // group identities: w == instance_z, h == instance_h, s1 + s2 == s3
            ok &= G1X::equal(G1X::from_affine(load_g1(A + A_W)), G1X::from_affine(load_g1(A + A_DYN + 384)));
            ok &= G1X::equal(G1X::from_affine(load_g1(A + A_H)), G1X::from_affine(load_g1(A + A_DYN + 448)));
            const G1X s12 = G1X::add_affine(G1X::from_affine(load_g1(A + A_WIRES)), load_g1(A + A_WIRES + 64));
            ok &= G1X::equal(s12, G1X::from_affine(load_g1(A + A_WIRES + 128)));
            // h + [public]_h == 0 (dynaverse.rs:1008-1015) when the proof has no
            // delta (kind 0); [public]_h = the side slots' value before the update
            // plus the public differences (a fresh anchor: zero plus the MSM of
            // all public inputs)
            const G1X pub = G1X::add_affine(G1X::from_affine(load_g1(r + SIDE_PUB)), load_g1(r + SIDE_PDIFF));
            if (J.kind == 0) ok &= G1X::add(G1X::add_affine(G1X::inf(), load_g1(A + A_H)), pub).is_inf();
            store_g1(r + SIDE_PUBNEW, pub.to_affine());
        }
    } else {
        const uint32_t aff2 = V_COUNT + J.fresh, unaff2 = aff2 + 1, us5 = aff2 + 2;
        if (lane == 7) {
            const G1A aff1 = load_g1(r + D_AFF1), unaff1 = load_g1(r + D_UNAFF1);
            Emit e = at(TAIL_TERMS);
            e.t(load_g1(r + D_PZQ), V_PZD); e.t(load_g1(r + D_W).neg(), V_G2);
            e.t(aff1, V_G2); e.t(g1.neg(), aff2);
            e.t(unaff1, V_G2); e.t(g1.neg(), unaff2);
            e.t(aff1, unaff2); e.t(mvg1.neg(), V_G2);
            // the local multiplication equation: ru[1] (lane 9), g1, ru[0] (lane 8), ru[2] (lane 10), quotient
            e.k = TAIL_TERMS + 9;
            e.t(g1.neg(), us5);
            e.k = TAIL_TERMS + 12;
            e.t(load_g1(r + D_LQ).neg(), aff2);
        } else if (lane <= 10) {
            // ru[i] = anchor local + changed local of wire s4 + i
            const uint32_t i = lane - 8;
            const G1A ru = g1_add(load_g1(r + D_ALOC + 64 * i), load_g1(r + D_CLOC + 64 * i));
            const uint32_t pos[3] = {TAIL_TERMS + 10, TAIL_TERMS + 8, TAIL_TERMS + 11};
            Emit e = at(pos[i]);
            if (i == 0) e.t(ru, us5);
            else if (i == 1) e.t(ru, V_G2);
            else e.t(ru.neg(), V_G2);
        } else if (lane <= 13) {
            // the openings of wire s4 + i against the affected and unaffected sets
            const uint32_t i = lane - 11;
            const G1A aw = load_g1(A + A_WIRES + 64 * (3 + i)), chw = load_g1(r + D_WIRES + 64 * (3 + i));
            Emit e = at(TAIL_TERMS + 13 + 6 * i);
            e.t(load_g1(r + D_AOPEN + 64 * i), aff2); e.t(g1_sub(aw, load_g1(r + D_ALOC + 64 * i)).neg(), V_G2);
            e.t(load_g1(r + D_COPEN + 64 * i), aff2); e.t(g1_sub(chw, load_g1(r + D_CLOC + 64 * i)).neg(), V_G2);
            e.t(load_g1(r + D_UZERO + 64 * i), unaff2); e.t(chw.neg(), V_G2);
        } else if (lane == 14) {
            ok &= G1X::equal(G1X::from_affine(load_g1(r + D_W)), G1X::from_affine(load_g1(r + D_DYN + 384)));
            ok &= G1X::equal(G1X::from_affine(load_g1(r + D_H)), G1X::from_affine(load_g1(r + D_DYN + 448)));
            const G1X s12 = G1X::add_affine(G1X::from_affine(load_g1(r + D_WIRES)), load_g1(r + D_WIRES + 64));
            ok &= G1X::equal(s12, G1X::from_affine(load_g1(r + D_WIRES + 128)));
            // anchor h + changed h + [public]_h == 0 (session.rs:127-131), with
            // [public]_h = the session's value plus this update's public differences
            const G1X pub_new = G1X::add_affine(G1X::from_affine(load_g1(r + SIDE_PUB)), load_g1(r + SIDE_PDIFF));
            G1X sum = G1X::add_affine(G1X::from_affine(load_g1(A + A_H)), load_g1(r + D_H));
            sum = G1X::add(sum, pub_new);
            ok &= sum.is_inf();
            store_g1(r + SIDE_PUBNEW, pub_new.to_affine());
        }
    }
    if (!ok) atomicOr(status + J.status, 8u);
}

// ================================================================ host: parameters
struct Params {
    uint64_t id = 0;
    uint32_t n = 0, m = 0, logn = 0;
    uint64_t fam_off[F_COUNT + 1] = {};
    uint64_t fam2_off[F2_COUNT + 1] = {};
    DevBuf srs, table, srs2, table2;  // Montgomery affine bases; c = 8 window multiples
    DevBuf table_dense;               // c = 16 window multiples of KZG bases [0, n)
    DevBuf wpow, inv1m;               // w^k, 1/(1 - w^k) (Montgomery)
    DevBuf vk2;                       // V_COUNT Montgomery G2 points
    DevBuf vk_lines, vk_inf;          // their Miller-loop lines, prepared once
    DevBuf consts;                    // canonical: [1]G1 | [X^n - 1]G1 | [X^n - 1]G2
    uint8_t vk2_bytes[V_COUNT][128] = {};
    uint8_t g1[64] = {}, mvg1[64] = {};
    uint32_t rebuild_interval = 1;
    hf::Fr n_m{}, ninv_m{};
    uint64_t footprint = 0;
};

uint64_t ceil_sqrt(uint64_t n) {  // dynaverse.rs:826-833
    uint64_t root = 1;
    while (root < n / root || (root == n / root && n % root != 0)) ++root;
    return root;
}

// sigma of ToyCircuit (toy_circuit.rs:17-27), an involution
uint32_t sigma_of(uint32_t n, uint32_t i) {
    if (i < n) return 6 * n + i;
    if (i >= 6 * n && i < 7 * n) return i - 6 * n;
    if (i >= 2 * n && i < 3 * n) return i + n;
    if (i >= 3 * n && i < 4 * n) return i - n;
    return i;
}

uint64_t params_bytes(uint64_t n) {
    const uint64_t rows = 100 * n, rows2 = 2 * n;
    return rows * 64 * (1 + TW) + n * 64 * TWD + rows2 * 128 * (1 + TW) + 2 * n * 32 + V_COUNT * 128 + 256;
}

// ================================================================ host: sessions and jobs
struct Session {
    uint64_t id = 0;
    Params* P = nullptr;
    uint32_t n = 0;
    // The current witness and instance.  The anchor's witness is not kept:
    // it is current minus `delta`, the nonzero differences by witness index.
    std::vector<Canon> pub, current;
    std::map<uint32_t, Canon> delta;
    std::vector<uint8_t> anchor_bytes;
    std::vector<uint8_t> proof;
    uint64_t anchor_generation = 0, generation = 0;
    uint8_t public_h[64] = {};
    DevBuf d_anchor, d_coef;  // anchor proof bytes; s4 | s5 | s6 coefficients
    uint64_t footprint = 0;
};

hf::Fr as_fr(const Canon& c) {
    hf::Fr r;
    memcpy(r.v, c.data(), 32);
    return r;
}

// The anchor's value at witness index i (current less the recorded difference).
Canon anchor_value(const Session& S, uint64_t i) {
    const auto it = S.delta.find((uint32_t)i);
    if (it == S.delta.end()) return S.current[i];
    const hf::Fr v = hf::sub(as_fr(S.current[i]), as_fr(it->second));
    Canon c;
    memcpy(c.data(), v.v, 32);
    return c;
}

struct Request {
    uint64_t ticket = 0, session = 0, submit_ns = 0;
    std::vector<uint64_t> idx, pidx;
    std::vector<Canon> vals, pvals;
};

struct Outcome {
    bool ready = false;
    int status = 0;
    std::string error;
    std::vector<uint8_t> proof;
    DvgpuDynaverseResult res{};
};

// One update of a batch after the host's bookkeeping (session.rs:51-109).
struct Job {
    Request* req = nullptr;
    Session* S = nullptr;
    bool rebuild = false;
    uint64_t generation = 0;
    std::map<uint64_t, Canon> edits, pedits;   // canonical new values
    std::map<uint32_t, Canon> delta;           // the new anchor differences
    // results
    bool ok = false;
    std::string error;
    std::vector<uint8_t> proof;
    uint8_t public_h[64] = {};
    std::vector<uint8_t> anchor_bytes;
    DevBuf new_anchor, new_coef;  // rebuild: replacement device state
};

// Host staging of one batch: descriptor blobs uploaded with one copy.
struct Stager {
    std::vector<uint8_t> h;
    size_t add(const void* p, size_t bytes) {
        const size_t off = (h.size() + 255) & ~size_t(255);
        h.resize(off + std::max<size_t>(bytes, 1));
        if (bytes) memcpy(h.data() + off, p, bytes);
        return off;
    }
    template <class T>
    size_t add(const std::vector<T>& v) {
        return add(v.data(), v.size() * sizeof(T));
    }
};

// One MSM launch under construction: segments, sets and output offsets.
struct MsmBuild {
    std::vector<SetDesc> segs;
    std::vector<uint32_t> seg_off{0}, set_off{0};
    std::vector<uint64_t> out_off;
    uint32_t terms = 0;
    void seg(uint32_t kind, uint64_t count, uint64_t row0, uint64_t sc0, uint64_t list) {
        if (!count) return;
        segs.push_back({kind, (uint32_t)count, (uint32_t)row0, (uint32_t)sc0, (uint32_t)list, 0});
        terms += (uint32_t)count;
        seg_off.push_back(terms);
    }
    void end(uint64_t out) {
        const uint32_t k = terms - set_off.back();
        set_off.push_back(terms);
        out_off.push_back(out);
        // algorithmic work of a k-term MSM: min over c of ceil(254/c) (10 k + 14 2^c) field
        // multiplications (XYZZ mixed additions and bucket reduction)
        if (k) {
            double best = 1e300;
            for (int c = 1; c <= 24; ++c)
                best = std::min(best, (double)((254 + c - 1) / c) * (10.0 * k + 14.0 * (double)(1u << c)));
            fme += best;
        }
    }
    double fme = 0;  // G1 field multiplications (x3 for G2 sets)
    size_t sets() const { return out_off.size(); }
    struct Dev {
        size_t segs, seg_off, set_off, out_off;
    } at{};
    void stage(Stager& s) {
        at.segs = s.add(segs);
        at.seg_off = s.add(seg_off);
        at.set_off = s.add(set_off);
        at.out_off = s.add(out_off);
    }
};

// The equation term counts of an anchor / delta verification, in order.
const std::vector<uint32_t>& eq_terms(bool delta) {
    static const std::vector<uint32_t> a = [] {
        std::vector<uint32_t> v = {5, 2, 2, 2};
        for (int t = 0; t < 6; ++t) v.insert(v.end(), {3, 2, 2, 2, 2});
        v.insert(v.end(), {2, 2, 3});
        return v;
    }();
    static const std::vector<uint32_t> d = [] {
        std::vector<uint32_t> v = {5, 2, 2, 2};
        for (int t = 0; t < 6; ++t) v.insert(v.end(), {3, 2, 2, 2, 2});
        v.insert(v.end(), {2, 2, 2, 2, 2, 3});
        for (int i = 0; i < 3; ++i) v.insert(v.end(), {2, 2, 2});
        return v;
    }();
    return delta ? d : a;
}

class Engine {
public:
    Engine(uint64_t budget, uint32_t max_batch) : budget_(budget), max_batch_(std::max<uint32_t>(1, max_batch)) {
        DV_CUDA(cudaGetDevice(&device_));
        worker_ = std::thread([this] { loop(); });
        run([this] {
            b_ = std::make_unique<Backend>();
            b_->device = device_;
            DV_CUDA(cudaStreamCreateWithFlags(&b_->stream, cudaStreamNonBlocking));
            st_ = b_->stream;
            DV_CUDA(cudaStreamCreateWithFlags(&st2_, cudaStreamNonBlocking));
            DV_CUDA(cudaStreamCreateWithFlags(&st3_, cudaStreamNonBlocking));
            DV_CUDA(cudaEventCreateWithFlags(&ev_fields_, cudaEventDisableTiming));
            DV_CUDA(cudaEventCreateWithFlags(&ev_g2_, cudaEventDisableTiming));
            DV_CUDA(cudaEventCreateWithFlags(&ev_start_, cudaEventDisableTiming));
            DV_CUDA(cudaEventCreateWithFlags(&ev_m1_, cudaEventDisableTiming));
            // phase events of the G1 workspace: the dense MSM, its last user in
            // a batch, leaves its accumulation time there for the stats
            for (auto& e : ws1_.timeline.ev) DV_CUDA(cudaEventCreate(&e));
            for (auto& e : ws1_.timeline.acc_ev) DV_CUDA(cudaEventCreate(&e));
            ws1_.timeline.enabled = true;
        });
    }
    ~Engine() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
    }

    // ------------------------------------------------------------ API (any thread)
    uint64_t params_create(uint64_t n, const uint8_t* tx, const uint8_t* ty) {
        uint64_t id = 0;
        run([&] { id = build_params(n, tx, ty); });
        return id;
    }
    void params_destroy(uint64_t id) {
        run([&] {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = params_.find(id);
            if (it == params_.end()) throw InvalidArgument("unknown parameters");
            for (auto& s : sessions_)
                if (s.second->P == it->second.get()) throw InvalidArgument("parameters have open sessions");
            resident_ -= it->second->footprint;
            params_.erase(it);
        });
    }
    void params_info(uint64_t id, DvgpuDynaverseParamsInfo* out) {
        run([&] {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = params_.find(id);
            if (it == params_.end()) throw InvalidArgument("unknown parameters");
            const Params& P = *it->second;
            memset(out, 0, sizeof(*out));
            out->n = P.n;
            out->m = P.m;
            out->rebuild_interval = P.rebuild_interval;
            out->resident_bytes = P.footprint;
            memcpy(out->g1_generator, P.g1, 64);
            memcpy(out->multiplication_vanishing_g1, P.mvg1, 64);
            for (int i = 0; i < V_COUNT; ++i) memcpy(out->vk_g2[i], P.vk2_bytes[i], 128);
        });
    }
    uint64_t open_session(uint64_t pid, const uint8_t* pub, const uint8_t* witness, uint8_t* proof) {
        uint64_t id = 0;
        run([&] { id = open_impl(pid, pub, witness, proof); });
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
            give(it->second->d_coef);  // kept for the next session or re-anchor
            give(it->second->d_anchor);
            sessions_.erase(it);
        });
    }
    void session_state(uint64_t id, uint8_t* witness, uint8_t* pub, uint8_t* proof, uint64_t* anchor_distance) {
        run([&] {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = sessions_.find(id);
            if (it == sessions_.end()) throw InvalidArgument("unknown session");
            const Session& S = *it->second;
            if (witness) memcpy(witness, S.current.data(), 32 * S.current.size());
            if (pub) memcpy(pub, S.pub.data(), 32 * S.pub.size());
            if (proof) memcpy(proof, S.proof.data(), PROOF_BYTES);
            if (anchor_distance) *anchor_distance = S.delta.size();
        });
    }
    uint64_t submit(uint64_t session, const uint64_t* idx, const uint8_t* vals, size_t k, const uint64_t* pidx,
                    const uint8_t* pvals, size_t pk) {
        Request r;
        r.submit_ns = now_ns();
        r.session = session;
        r.idx.assign(idx, idx + k);
        r.pidx.assign(pidx, pidx + pk);
        r.vals.resize(k);
        r.pvals.resize(pk);
        for (size_t j = 0; j < k; ++j) {
            if (!canon_ok(vals + 32 * j)) throw InvalidArgument("non-canonical update value");
            memcpy(r.vals[j].data(), vals + 32 * j, 32);
        }
        for (size_t j = 0; j < pk; ++j) {
            if (!canon_ok(pvals + 32 * j)) throw InvalidArgument("non-canonical public input value");
            memcpy(r.pvals[j].data(), pvals + 32 * j, 32);
        }
        std::lock_guard<std::mutex> lk(mu_);
        if (!sessions_.count(session)) throw InvalidArgument("unknown session");
        r.ticket = next_ticket_++;
        outcomes_[r.ticket];
        queue_.push_back(std::move(r));
        cv_.notify_all();
        return queue_.back().ticket;
    }
    void wait(uint64_t ticket, uint8_t* proof, DvgpuDynaverseResult* res) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = outcomes_.find(ticket);
        if (it == outcomes_.end()) throw InvalidArgument("unknown ticket");
        done_cv_.wait(lk, [&] { return it->second.ready; });
        Outcome o = std::move(it->second);
        outcomes_.erase(it);
        lk.unlock();
        if (o.status == -1) throw InvalidArgument(o.error);
        if (o.status != 0) throw CudaFailure(o.error);
        if (proof) memcpy(proof, o.proof.data(), PROOF_BYTES);
        if (res) *res = o.res;
    }
    void verify(uint64_t pid, const uint8_t* pub, const uint8_t* proof, uint8_t* accepted) {
        run([&] { *accepted = verify_impl(pid, pub, proof) ? 1 : 0; });
    }
    void set_max_batch(uint32_t m) {
        std::lock_guard<std::mutex> lk(mu_);
        max_batch_ = std::max<uint32_t>(1, m);
    }
    DvgpuDynaverseStats stats() {
        std::lock_guard<std::mutex> lk(mu_);
        DvgpuDynaverseStats s{};
        s.requests = stat_requests_;
        s.batches = stat_batches_;
        s.sessions = sessions_.size();
        s.resident_bytes = resident_;
        s.budget_bytes = budget_;
        s.max_batch = max_batch_;
        s.largest_batch = stat_largest_;
        s.busy_ns = stat_busy_ns_;
        s.pending = queue_.size();
        s.sparse_proofs = stat_sparse_;
        s.rebuilds = stat_rebuilds_;
        s.launches = stat_launches_;
        s.msm_fme = stat_fme_.load();
        s.device_wait_ns = stat_wait_ns_.load();
        s.dense_accum_ns = stat_dense_ns_.load();
        s.dense_accum_adds = stat_dense_adds_.load();
        s.allocations = stat_allocs_;
        s.allocation_ns = stat_alloc_ns_;
        s.enqueue_ns = stat_enqueue_ns_.load();
        for (int i = 0; i < 3; ++i) (&s.slowest_alloc_ns)[i] = __atomic_load_n(slowest_alloc() + i, __ATOMIC_RELAXED);
        s.host_ns = s.busy_ns > s.device_wait_ns ? s.busy_ns - s.device_wait_ns : 0;
        return s;
    }

private:
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
            std::vector<Session*> sess(batch.size(), nullptr);
            for (size_t r = 0; r < batch.size(); ++r) {
                auto it = sessions_.find(batch[r].session);
                if (it != sessions_.end()) sess[r] = it->second.get();
            }
            lk.unlock();
            const uint64_t t0 = now_ns();
            const uint64_t l0 = __atomic_load_n(&launch_counter(), __ATOMIC_RELAXED);
            const uint64_t a0 = __atomic_load_n(&alloc_counter(), __ATOMIC_RELAXED);
            const uint64_t an0 = __atomic_load_n(&alloc_ns_counter(), __ATOMIC_RELAXED);
            std::vector<Outcome> outs(batch.size());
            process(batch, sess, outs);
            const uint64_t t1 = now_ns();
            lk.lock();
            for (size_t r = 0; r < batch.size(); ++r) {
                Outcome& o = outcomes_[batch[r].ticket];
                o = std::move(outs[r]);
                o.res.submit_ns = batch[r].submit_ns;
                o.res.start_ns = t0;
                o.res.done_ns = t1;
                o.res.batch_requests = (uint32_t)batch.size();
                o.res.batch_id = (uint32_t)stat_batches_;
                o.ready = true;
            }
            stat_requests_ += batch.size();
            stat_batches_++;
            stat_largest_ = std::max<uint64_t>(stat_largest_, batch.size());
            stat_busy_ns_ += t1 - t0;
            stat_launches_ += __atomic_load_n(&launch_counter(), __ATOMIC_RELAXED) - l0;
            stat_allocs_ += __atomic_load_n(&alloc_counter(), __ATOMIC_RELAXED) - a0;
            stat_alloc_ns_ += __atomic_load_n(&alloc_ns_counter(), __ATOMIC_RELAXED) - an0;
            done_cv_.notify_all();
        }
        ws1_.timeline.enabled = false;
        for (auto& e : ws1_.timeline.ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : ws1_.timeline.acc_ev)
            if (e) cudaEventDestroy(e);
        for (auto& sp : spare_) cudaFree(sp.first);
        spare_.clear();
        for (cudaEvent_t e : {ev_fields_, ev_g2_, ev_start_, ev_m1_})
            if (e) cudaEventDestroy(e);
        if (st2_) cudaStreamDestroy(st2_);
        if (st3_) cudaStreamDestroy(st3_);
        b_.reset();
    }

    // ------------------------------------------------------------ parameters
    uint64_t build_params(uint64_t n, const uint8_t* txb, const uint8_t* tyb);
    // ------------------------------------------------------------ pipelines
    template <class F>
    void run_msm(MsmWorkspace& ws, const Affine<F>* table, MsmBuild& mb, const uint8_t* d_stage,
                 const uint32_t* lrow, const uint32_t* lsc, const Fr* arena, uint8_t* out, uint32_t* d_err,
                 DevBuf& tpoint, DevBuf& tscalar, cudaStream_t st, int tc = TC, int tw = TW);
    // The batch's pairing lines: the verifying key's (prepared with the
    // parameters), then the nfresh own G2 points at q + V_COUNT, prepared on st.
    void prepare_lines(Params& P, const G2A* q, uint64_t nfresh, cudaStream_t st);
    void run_anchor(Params& P, const std::vector<Canon>& w, const std::vector<Canon>& pub, Job& job);
    void run_sparse(Params& P, std::vector<Job*>& jobs);
    void run_verify(Params& P, uint32_t njobs, uint64_t nfresh, uint64_t terms, uint64_t eqs, const VerifyJob* d_jobs,
                    const uint64_t* d_off, uint8_t* d_verdicts, uint32_t* d_status);
    void upload(Stager& stg);
    uint64_t open_impl(uint64_t pid, const uint8_t* pub, const uint8_t* witness, uint8_t* proof);
    bool verify_impl(uint64_t pid, const uint8_t* pub, const uint8_t* proof);
    void process(std::vector<Request>& batch, std::vector<Session*>& sess, std::vector<Outcome>& outs);
    void stage_job(Request& r, Session* S, Job& job);

    int device_ = 0;
    std::unique_ptr<Backend> b_;
    cudaStream_t st_ = nullptr;
    uint64_t budget_, resident_ = 0;
    uint32_t max_batch_;
    MsmWorkspace ws1_, ws2_;
    NttBatch nb_fwd_, nb_inv_, nb_r1_, nb_r2_, nb_r3_;
    DevBuf stage_, arena_, scr_, out_, status_, verdicts_, tpoint_, tscalar_, tpoint2_, tscalar2_, lrow_, lsc_,
        terms_p_, terms_q_, g2q_, lines_, qinf_, tmp_, tmp2_, err_;
    // The G2 side of an update batch (its MSM, then preparing the fresh G2
    // points for the pairings) runs on st2_ beside the dense G1 work on st_;
    // the linear fields' MSM (m1), which only the record copies and the
    // verification read, runs on st3_ from the start of the batch, then the
    // affected-set MSM (m2) once the field rows exist, beside the dense MSM.
    cudaStream_t st2_ = nullptr, st3_ = nullptr;
    cudaEvent_t ev_fields_ = nullptr, ev_g2_ = nullptr, ev_start_ = nullptr, ev_m1_ = nullptr;
    MsmWorkspace ws3_;
    DevBuf tpoint3_, tscalar3_;
    bool quot_smem_ = false;
    PinnedBuf pstage_, pstage2_, parena_, pout_;

    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    bool stop_ = false;
    std::deque<std::function<void()>> cmds_;
    std::deque<Request> queue_;
    std::map<uint64_t, std::unique_ptr<Params>> params_;
    std::map<uint64_t, std::unique_ptr<Session>> sessions_;
    std::map<uint64_t, Outcome> outcomes_;
    uint64_t next_id_ = 1, next_ticket_ = 1;
    uint64_t stat_requests_ = 0, stat_batches_ = 0, stat_largest_ = 0, stat_busy_ns_ = 0, stat_sparse_ = 0,
             stat_rebuilds_ = 0, stat_launches_ = 0;
    std::atomic<uint64_t> stat_fme_{0};  // written by the worker, read by stats()
    std::atomic<uint64_t> stat_wait_ns_{0}, stat_dense_ns_{0}, stat_dense_adds_{0};
    uint64_t stat_allocs_ = 0, stat_alloc_ns_ = 0;  // under mu_
    std::atomic<uint64_t> stat_enqueue_ns_{0};
    // Device buffers that re-anchors swap out of sessions and that closed
    // sessions leave (coefficients, anchor bytes), kept for the next
    // re-anchor or session: once the pool holds a batch's worth, neither
    // allocates nor frees (device allocation can take milliseconds and
    // freeing waits for the device).  At most SPARE_MAX buffers are kept.
    std::vector<std::pair<void*, size_t>> spare_;
    static constexpr size_t SPARE_MAX = 1024;
    void take(DevBuf& b, size_t bytes) {
        if (b.ptr && b.cap >= bytes) return;
        size_t best = spare_.size();  // the smallest spare that fits, so small sessions leave large buffers
        for (size_t i = 0; i < spare_.size(); ++i)
            if (spare_[i].second >= bytes && (best == spare_.size() || spare_[i].second < spare_[best].second))
                best = i;
        if (best < spare_.size()) {
            b.release();
            b.ptr = spare_[best].first;
            b.cap = spare_[best].second;
            spare_[best] = spare_.back();
            spare_.pop_back();
            return;
        }
        b.get(bytes);
    }
    void give(DevBuf& b) {
        if (!b.ptr) return;
        if (spare_.size() < SPARE_MAX) {
            spare_.push_back({b.ptr, b.cap});
            b.ptr = nullptr;
            b.cap = 0;
        } else {
            b.release();
        }
    }
    std::thread worker_;
};

// ================================================================ parameters (setup)
// DynaverseParams::setup_impl from explicit trapdoors (the reference samples
// them, srs.rs:158-178, and discards them after setup).
uint64_t Engine::build_params(uint64_t n, const uint8_t* txb, const uint8_t* tyb) {
    using namespace hf;
    if (!n || (n & (n - 1)) || n > (1u << 17)) throw InvalidArgument("n must be a power of two in 1..2^17");
    if (!canon_ok(txb) || !canon_ok(tyb)) throw InvalidArgument("non-canonical trapdoor");
    const uint64_t m = 8 * n, six = 6 * n, seven = 7 * n;
    const uint64_t need = params_bytes(n);
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (resident_ + need > budget_)
            throw InvalidArgument("parameters do not fit the HBM budget (" + std::to_string(resident_) + " + " +
                                  std::to_string(need) + " > " + std::to_string(budget_) + " bytes)");
    }
    Canon ctx, cty;
    memcpy(ctx.data(), txb, 32);
    memcpy(cty.data(), tyb, 32);
    const Fr tx = mont_of(ctx), ty = mont_of(cty), o = one();
    const Fr txm = pow_u64(tx, m), tym = pow_u64(ty, m), ty8 = pow_u64(ty, 8);
    if (is_zero(tx) || is_zero(ty) || eq(txm, o) || eq(tym, o) || eq(tx, ty))
        throw InvalidArgument("trapdoors must be nonzero, distinct and outside the domain");
    if (eq(tx, ty8)) throw InvalidArgument("consistency divisor vanishes");
    const Fr wm = root(m), wn = root(n);
    std::vector<Fr> pw(m);
    par_for(m, [&](uint64_t lo, uint64_t hi) {
        Fr p = pow_u64(wm, lo);
        for (uint64_t i = lo; i < hi; ++i) {
            pw[i] = p;
            p = mul(p, wm);
        }
    });
    const Fr inv_m = inv(from_u64(m)), inv_n = inv(from_u64(n));
    std::vector<Fr> dx(seven), dy(seven);
    par_for(seven, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            dx[i] = sub(tx, pw[i]);
            dy[i] = sub(ty, pw[i]);
        }
    });
    // z_in of each slice and I_x (consistency.rs:217-224, srs.rs:91-96)
    Fr zin[6], ix = o;
    for (int t = 0; t < 6; ++t) {
        zin[t] = o;
        for (uint64_t i = t * n; i < (t + 1) * n; ++i) zin[t] = mul(zin[t], dx[i]);
    }
    for (uint64_t i = six; i < m; ++i) ix = mul(ix, sub(tx, pw[i]));
    par_batch_inv(dx);
    par_batch_inv(dy);
    const Fr lxs = mul(sub(txm, o), inv_m), lys = mul(sub(tym, o), inv_m);
    std::vector<Fr> lx(seven), ly(seven), y(seven);
    par_for(seven, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            lx[i] = mul(mul(lxs, pw[i]), dx[i]);
            ly[i] = mul(mul(lys, pw[i]), dy[i]);
        }
    });
    par_for(seven, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) y[i] = sub(ly[i], ly[sigma_of((uint32_t)n, (uint32_t)i)]);
    });
    // u = sum lx_i y_i (y vanishes outside [0, 4n) and [6n, 7n), dynamo.rs:181-185)
    Fr u = zero();
    for (uint64_t i = 0; i < seven; ++i) u = add(u, mul(lx[i], y[i]));
    const Fr xv_inv = inv(sub(txm, o)), tx_inv = inv(tx);
    auto lagr = [&](const Fr& tau) {  // lagrange_values(tau, n) (setup.rs:48-61)
        std::vector<Fr> d(n), out(n);
        const Fr num = mul(sub(pow_u64(tau, n), o), inv_n);
        for (uint64_t j = 0; j < n; ++j) d[j] = sub(tau, pw[8 * j]);  // w_n^j = w_m^(8j)
        batch_inv(d.data(), n);
        for (uint64_t j = 0; j < n; ++j) out[j] = mul(mul(num, pw[8 * j]), d[j]);
        return out;
    };
    const std::vector<Fr> lsx = lagr(tx), cx = lagr(pow_u64(tx, 8)), cy = lagr(ty8);
    std::vector<Fr> sinv(n);
    for (uint64_t j = 0; j < n; ++j) sinv[j] = sub(tx, pw[8 * j]);
    batch_inv(sinv.data(), n);
    Fr zin_inv[6];
    for (int t = 0; t < 6; ++t) zin_inv[t] = inv(zin[t]);
    const Fr xy_inv = inv(sub(tx, ty)), sub_inv = inv(sub(tx, ty8)), ix_inv = inv(ix);
    std::vector<Fr> txp(n);
    txp[0] = o;
    for (uint64_t j = 1; j < n; ++j) txp[j] = mul(txp[j - 1], tx);

    auto P = std::make_unique<Params>();
    P->n = (uint32_t)n;
    P->m = (uint32_t)m;
    while ((1ull << P->logn) < n) ++P->logn;
    uint64_t off = 0;
    for (int f = 0; f < F_COUNT; ++f) {
        P->fam_off[f] = off;
        off += fam_size(f, n);
    }
    P->fam_off[F_COUNT] = off;
    const uint64_t rows = off;
    P->fam2_off[F2_LAG] = 0;
    P->fam2_off[F2_KZG] = n;
    P->fam2_off[F2_COUNT] = 2 * n;
    std::vector<Canon> sc(rows);
    auto put = [&](int f, uint64_t i, const Fr& v) { sc[P->fam_off[f] + i] = canon_of(v); };
    par_for(six, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) {
            const Fr common = mul(y[i], sub(lx[i], inv_m));
            put(F_LX, i, lx[i]);
            put(F_ALPHA, i, mul(mul(lx[i], sub(u, y[i])), xv_inv));
            put(F_BETA, i, mul(common, tx_inv));
            put(F_H, i, mul(txm, y[i]));
            put(F_Z, i, mul(tym, lx[i]));
            put(F_B, i, mul(common, tx));
            for (int t = 0; t < 6; ++t) {
                Fr v = lx[i];
                if (i >= t * n && i < (t + 1) * n) v = sub(v, cx[i - t * n]);
                put(F_QAC0 + t, i, mul(v, zin_inv[t]));
            }
            put(F_ADEG, i, mul(lx[i], tym));
            put(F_PQ, i, mul(lx[i], ix_inv));
        }
    });
    for (uint64_t i = 0; i < seven; ++i) put(F_LY, i, ly[i]);
    for (uint64_t j = 0; j < n; ++j) {
        put(F_LAG, j, lsx[j]);
        put(F_OPENU, j, mul(sub(lsx[j], o), sinv[j]));
        put(F_QCD, j, mul(sub(cx[j], cy[j]), xy_inv));
        put(F_QBD, j, mul(sub(lsx[j], cy[j]), sub_inv));
        put(F_D, j, cy[j]);
        put(F_BDEG, j, mul(lsx[j], tym));
        put(F_DDEG, j, mul(cy[j], txm));
        put(F_KZG, j, txp[j]);
        put(F_PUBH, j, sub(ly[six + j], ly[j]));
    }
    std::vector<Canon> sc2(2 * n);
    for (uint64_t j = 0; j < n; ++j) {
        sc2[j] = canon_of(lsx[j]);
        sc2[n + j] = canon_of(txp[j]);
    }
    const Fr zn = sub(pow_u64(tx, n), o);
    std::vector<Canon> vks(V_COUNT);
    vks[V_U] = canon_of(u);
    vks[V_XM1] = canon_of(sub(txm, o));
    vks[V_X] = canon_of(tx);
    vks[V_INVM] = canon_of(inv_m);
    vks[V_YM1] = canon_of(sub(tym, o));
    vks[V_YM] = canon_of(tym);
    vks[V_XM] = canon_of(txm);
    vks[V_X2] = canon_of(mul(tx, tx));
    vks[V_G2] = canon_of(o);
    for (int t = 0; t < 6; ++t) vks[V_ZIN0 + t] = canon_of(zin[t]);
    vks[V_XMY] = canon_of(sub(tx, ty));
    vks[V_XMLY] = canon_of(sub(tx, ty8));
    vks[V_PZD] = canon_of(ix);
    vks[V_MD] = canon_of(zn);
    const std::vector<Canon> g1s = {canon_of(o), canon_of(zn)};
    // field tables of the n-point domain
    std::vector<Fr> wp(n), i1m(n);
    for (uint64_t k = 0; k < n; ++k) wp[k] = pw[8 * k];
    i1m[0] = zero();
    for (uint64_t k = 1; k < n; ++k) i1m[k] = sub(o, wp[k]);
    if (n > 1) batch_inv(i1m.data() + 1, n - 1);
    P->rebuild_interval = (uint32_t)ceil_sqrt(n);
    P->n_m = from_u64(n);
    P->ninv_m = inv_n;

    // device: fixed-base points, Montgomery bases, window tables
    const cudaStream_t st = st_;
    uint32_t* bad = err_.as<uint32_t>(4);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, 16, st));
    {
        uint8_t* d_sc = tmp_.as<uint8_t>(rows * 32);
        uint8_t* d_pt = tmp2_.as<uint8_t>(rows * 64);
        DV_CUDA(cudaMemcpyAsync(d_sc, sc.data(), rows * 32, cudaMemcpyHostToDevice, st));
        fixed_base_launch(b_->fixed_base, d_sc, rows, 0, d_pt, bad, st);
        G1A* srs = P->srs.as<G1A>(rows);
        convert_points<Fq>(d_pt, srs, rows, bad + 1, st);
        msm_precompute<Fq>(srs, rows, TC, TW, P->table.as<G1A>(rows * TW), st);
        msm_precompute<Fq>(srs + P->fam_off[F_KZG], n, TCD, TWD, P->table_dense.as<G1A>(n * TWD), st);
        DV_CUDA(cudaStreamSynchronize(st));
    }
    {
        const uint64_t r2 = 2 * n;
        uint8_t* d_sc = tmp_.as<uint8_t>(r2 * 32);
        uint8_t* d_pt = tmp2_.as<uint8_t>(r2 * 128);
        DV_CUDA(cudaMemcpyAsync(d_sc, sc2.data(), r2 * 32, cudaMemcpyHostToDevice, st));
        fixed_base_launch(b_->fixed_base, d_sc, r2, 1, d_pt, bad, st);
        G2A* srs2 = P->srs2.as<G2A>(r2);
        convert_points<Fq2>(d_pt, srs2, r2, bad + 2, st);
        msm_precompute<Fq2>(srs2, r2, TC, TW, P->table2.as<G2A>(r2 * TW), st);
        DV_CUDA(cudaStreamSynchronize(st));
    }
    {
        uint8_t* d_sc = tmp_.as<uint8_t>(32 * (V_COUNT + 2));
        uint8_t* d_pt = tmp2_.as<uint8_t>(128 * V_COUNT + 128);
        DV_CUDA(cudaMemcpyAsync(d_sc, vks.data(), 32 * V_COUNT, cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaMemcpyAsync(d_sc + 32 * V_COUNT, g1s.data(), 64, cudaMemcpyHostToDevice, st));
        fixed_base_launch(b_->fixed_base, d_sc, V_COUNT, 1, d_pt, bad, st);
        fixed_base_launch(b_->fixed_base, d_sc + 32 * V_COUNT, 2, 0, d_pt + 128 * V_COUNT, bad, st);
        convert_points<Fq2>(d_pt, P->vk2.as<G2A>(V_COUNT), V_COUNT, bad + 3, st);
        pairing_prepare_device(P->vk2.view<G2A>(), V_COUNT, P->vk_lines.as<uint8_t>(V_COUNT * pairing_prepared_bytes()),
                               P->vk_inf.as<uint32_t>(V_COUNT), st);
        uint8_t* consts = P->consts.as<uint8_t>(256);
        DV_CUDA(cudaMemcpyAsync(consts, d_pt + 128 * V_COUNT, 128, cudaMemcpyDeviceToDevice, st));
        DV_CUDA(cudaMemcpyAsync(consts + 128, d_pt + 128 * V_MD, 128, cudaMemcpyDeviceToDevice, st));
        DV_CUDA(cudaMemcpyAsync(P->vk2_bytes, d_pt, 128 * V_COUNT, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaMemcpyAsync(P->g1, d_pt + 128 * V_COUNT, 64, cudaMemcpyDeviceToHost, st));
        DV_CUDA(cudaMemcpyAsync(P->mvg1, d_pt + 128 * V_COUNT + 64, 64, cudaMemcpyDeviceToHost, st));
    }
    DV_CUDA(cudaMemcpyAsync(P->wpow.as<uint8_t>(32 * n), wp.data(), 32 * n, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(P->inv1m.as<uint8_t>(32 * n), i1m.data(), 32 * n, cudaMemcpyHostToDevice, st));
    uint32_t hbad[4];
    DV_CUDA(cudaMemcpyAsync(hbad, bad, 16, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < 4; ++i)
        if (hbad[i] != 0xffffffffu) throw CudaFailure("parameter setup produced an invalid point");
    tmp_.release();
    tmp2_.release();
    P->footprint = need;
    std::lock_guard<std::mutex> lk(mu_);
    P->id = next_id_++;
    resident_ += need;
    const uint64_t id = P->id;
    params_[id] = std::move(P);
    return id;
}

// ================================================================ pipelines
template <class F>
void Engine::run_msm(MsmWorkspace& ws, const Affine<F>* table, MsmBuild& mb, const uint8_t* d_stage,
                     const uint32_t* lrow, const uint32_t* lsc, const Fr* arena, uint8_t* out, uint32_t* d_err,
                     DevBuf& tpoint, DevBuf& tscalar, cudaStream_t st, int tc, int tw) {
    if (!mb.sets() || !mb.terms) return;  // no terms: every field stays zero bytes (infinity)
    uint32_t* tp = tpoint.as<uint32_t>(mb.terms);
    uint32_t* ts = tscalar.as<uint32_t>(mb.terms);
    k_dv_expand<<<(mb.terms + 255) / 256, 256, 0, st>>>(
        mb.terms, (uint32_t)mb.segs.size(), reinterpret_cast<const uint32_t*>(d_stage + mb.at.seg_off),
        reinterpret_cast<const SetDesc*>(d_stage + mb.at.segs), lrow, lsc, tp, ts);
    DV_LAUNCH();
    const MsmPrecomp<F> pre{table, tc, tw};
    const uint32_t sets = (uint32_t)mb.sets();
    const MsmPlan plan = msm_plan_batch<F>(sets, 0, mb.terms, 0, &pre);
    SetMap map{reinterpret_cast<const uint32_t*>(d_stage + mb.at.set_off), nullptr, sets, 0, tp, ts};
    msm_enqueue<F>(ws, nullptr, reinterpret_cast<const uint32_t*>(arena), map, mb.terms, plan, &pre, d_err, st);
    k_dv_affine<F><<<(sets + 127) / 128, 128, 0, st>>>(ws.windows.view<XYZZ<F>>(), sets,
                                                        reinterpret_cast<const uint64_t*>(d_stage + mb.at.out_off),
                                                        out);
    DV_LAUNCH();
}

// Montgomery affine G1 point from canonical bytes (host).
G1A host_g1(const uint8_t* b) {
    G1A r;
    memset(&r, 0, sizeof(r));
    uint64_t x[4], y[4];
    memcpy(x, b, 32);
    memcpy(y, b + 32, 32);
    bool zero = true;
    for (int i = 0; i < 64; ++i) zero &= b[i] == 0;
    if (zero) return r;
    const dvh::Fq hx = dvh::from_canonical(x), hy = dvh::from_canonical(y);
    static_assert(sizeof(dvh::Fq) == 32, "host/device field layout");
    memcpy(&r.x, &hx, 32);
    memcpy(&r.y, &hy, 32);
    return r;
}

// Builds and checks the equations of njobs staged verification jobs: term
// arrays, the G2 array (the verifying key, then the jobs' own points), one
// pairing check.  Verdict bytes (one per equation) land at d_verdicts.
void Engine::run_verify(Params& P, uint32_t njobs, uint64_t nfresh, uint64_t terms, uint64_t eqs,
                        const VerifyJob* d_jobs, const uint64_t* d_off, uint8_t* d_verdicts, uint32_t* d_status) {
    G1A* p = terms_p_.as<G1A>(std::max<uint64_t>(1, terms));
    uint32_t* qi = terms_q_.as<uint32_t>(std::max<uint64_t>(1, terms));
    G2A* q = g2q_.as<G2A>(V_COUNT + nfresh);
    DV_CUDA(cudaMemcpyAsync(q, P.vk2.view<G2A>(), V_COUNT * sizeof(G2A), cudaMemcpyDeviceToDevice, st_));
    k_dv_fresh<<<(njobs + 31) / 32, 32, 0, st_>>>(d_jobs, njobs, q);
    DV_LAUNCH();
    k_dv_terms<<<dim3(njobs, TERM_PIECES), 32, 0, st_>>>(d_jobs, njobs, host_g1(P.g1), host_g1(P.mvg1), p, qi,
                                                         d_status);
    DV_LAUNCH();
    prepare_lines(P, q, nfresh, st_);
    pairing_check_prepared(*b_, p, terms, lines_.view<uint8_t>(), qinf_.view<uint32_t>(), qi, d_off, eqs, d_verdicts,
                           st_);
}

void Engine::prepare_lines(Params& P, const G2A* q, uint64_t nfresh, cudaStream_t st) {
    const uint64_t lb = pairing_prepared_bytes();
    uint8_t* lines = lines_.as<uint8_t>((V_COUNT + nfresh) * lb);
    uint32_t* qinf = qinf_.as<uint32_t>(V_COUNT + nfresh);
    DV_CUDA(cudaMemcpyAsync(lines, P.vk_lines.view<uint8_t>(), V_COUNT * lb, cudaMemcpyDeviceToDevice, st));
    DV_CUDA(cudaMemcpyAsync(qinf, P.vk_inf.view<uint32_t>(), 4 * V_COUNT, cudaMemcpyDeviceToDevice, st));
    pairing_prepare_device(q + V_COUNT, nfresh, lines + V_COUNT * lb, qinf + V_COUNT, st);
}

void Engine::upload(Stager& stg) {
    uint8_t* h = pstage_.as<uint8_t>(stg.h.size());
    memcpy(h, stg.h.data(), stg.h.size());
    uint8_t* d = stage_.as<uint8_t>(stg.h.size());
    DV_CUDA(cudaMemcpyAsync(d, h, stg.h.size(), cudaMemcpyHostToDevice, st_));
}

std::vector<uint64_t> eq_offsets(size_t jobs, bool delta) {
    std::vector<uint64_t> off{0};
    for (size_t j = 0; j < jobs; ++j)
        for (uint32_t c : eq_terms(delta)) off.push_back(off.back() + c);
    return off;
}

// The anchor proof of a witness (prove_anchor_traced, dynaverse.rs:149-248)
// and its verification (verify_anchor_with_checks and the public-input
// identity, dynaverse.rs:1018-1044, 1008-1015).  Results in `job`.
void Engine::run_anchor(Params& P, const std::vector<Canon>& w, const std::vector<Canon>& pub, Job& job) {
    const uint64_t n = P.n;
    const uint64_t W = 0, H = 6 * n, PB = 13 * n, Q = 14 * n, P0 = 15 * n, P1 = 17 * n, TOT = 19 * n;
    const cudaStream_t st = st_;
    Fr* arena = arena_.as<Fr>(TOT);
    take(job.new_coef, 3 * n * sizeof(Fr));
    take(job.new_anchor, ANCHOR_BYTES);
    Fr* coef = job.new_coef.view<Fr>();
    uint8_t* anc = job.new_anchor.view<uint8_t>();
    uint8_t* rec = out_.as<uint8_t>(JOB_BYTES);
    uint32_t* status = status_.as<uint32_t>(1);
    uint8_t* verd = verdicts_.as<uint8_t>(ANCHOR_EQS);
    uint32_t* err = err_.as<uint32_t>(2);
    Canon* hin = parena_.as<Canon>(7 * n);
    memcpy(hin, w.data(), 32 * 6 * n);
    memcpy(hin + 6 * n, pub.data(), 32 * n);
    DV_CUDA(cudaMemcpyAsync(arena + W, hin, 32 * 6 * n, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(arena + PB, hin + 6 * n, 32 * n, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemsetAsync(rec, 0, JOB_BYTES, st));
    DV_CUDA(cudaMemsetAsync(status, 0, 4, st));
    DV_CUDA(cudaMemsetAsync(err, 0xff, 8, st));
    k_dv_h<<<(unsigned)((7 * n + 255) / 256), 256, 0, st>>>(arena + W, (uint32_t)n, arena + H);
    DV_LAUNCH();
    // s4, s5, s6 coefficients (kept by the session for the anchor openings)
    for (int t = 0; t < 3; ++t)
        ntt_run(b_->ntt, reinterpret_cast<const uint8_t*>(arena + W + (3 + t) * n),
                reinterpret_cast<uint8_t*>(coef + t * n), (int)P.logn, NTT_INVERSE, st);
    // multiplication quotient (s4 s5 - s6) / (X^n - 1)
    const unsigned g2n = (unsigned)((2 * n + 255) / 256);
    k_dv_pad<<<g2n, 256, 0, st>>>(coef, n, arena + P0, 2 * n);
    DV_LAUNCH();
    k_dv_pad<<<g2n, 256, 0, st>>>(coef + n, n, arena + P1, 2 * n);
    DV_LAUNCH();
    ntt_run(b_->ntt, reinterpret_cast<const uint8_t*>(arena + P0), reinterpret_cast<uint8_t*>(arena + P0),
            (int)P.logn + 1, NTT_FORWARD, st);
    ntt_run(b_->ntt, reinterpret_cast<const uint8_t*>(arena + P1), reinterpret_cast<uint8_t*>(arena + P1),
            (int)P.logn + 1, NTT_FORWARD, st);
    k_dv_pmul<<<g2n, 256, 0, st>>>(arena + P0, arena + P1, 2 * n);
    DV_LAUNCH();
    ntt_run(b_->ntt, reinterpret_cast<const uint8_t*>(arena + P0), reinterpret_cast<uint8_t*>(arena + P0),
            (int)P.logn + 1, NTT_INVERSE, st);
    k_dv_mq<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(arena + P0, coef + 2 * n, (uint32_t)n, arena + Q, status);
    DV_LAUNCH();
    // every commitment of the anchor in one G1 launch and one G2 launch
    MsmBuild g1, g2;
    auto fo = [&](int f) { return P.fam_off[f]; };
    const uint64_t RA = REC_ANCHOR;
    for (int t = 0; t < 6; ++t) {
        g1.seg(0, n, fo(F_LAG), W + t * n, 0);
        g1.end(RA + A_WIRES + 64 * t);
    }
    g1.seg(0, 6 * n, fo(F_LX), W, 0);
    g1.end(RA + A_W);
    g1.seg(0, 7 * n, fo(F_LY), H, 0);
    g1.end(RA + A_H);
    const int dyf[5] = {F_ALPHA, F_BETA, F_H, F_Z, F_B};
    for (int k = 0; k < 5; ++k) {
        g1.seg(0, 6 * n, fo(dyf[k]), W, 0);
        g1.end(RA + A_DYN + 64 * k);
    }
    for (int t = 0; t < 6; ++t) {
        const uint64_t base = RA + A_CONS + 448 * t;
        g1.seg(0, 6 * n, fo(F_QAC0 + t), W, 0);
        g1.end(base);
        const int cf[3] = {F_QCD, F_QBD, F_D};
        for (int k = 0; k < 3; ++k) {
            g1.seg(0, n, fo(cf[k]), W + t * n, 0);
            g1.end(base + 64 * (1 + k));
        }
        if (t == 0) {
            g1.seg(0, 6 * n, fo(F_ADEG), W, 0);
            g1.end(base + 256);
        }
        g1.seg(0, n, fo(F_BDEG), W + t * n, 0);
        g1.end(base + 320);
        g1.seg(0, n, fo(F_DDEG), W + t * n, 0);
        g1.end(base + 384);
    }
    g1.seg(0, 6 * n, fo(F_PQ), W, 0);
    g1.end(RA + A_PZQ);
    g1.seg(0, n - 1, fo(F_KZG), Q, 0);
    g1.end(RA + A_MQ);
    g1.seg(0, n, fo(F_PUBH), PB, 0);
    g1.end(SIDE_PDIFF);
    g2.seg(0, n, P.fam2_off[F2_LAG], W + 4 * n, 0);
    g2.end(RA + A_S5G2);
    uint8_t* an = rec + RA;
    std::vector<CopyDesc> cp = {{an + A_DYN + 64 * DY_IZ, an + A_W, 64}, {an + A_DYN + 64 * DY_IH, an + A_H, 64}};
    for (int t = 1; t < 6; ++t) cp.push_back({an + A_CONS + 448 * t + 256, an + A_CONS + 256, 64});
    const VerifyJob vj{rec, an, 0, 0, 0, 0};
    const std::vector<uint64_t> off = eq_offsets(1, false);
    Stager stg;
    g1.stage(stg);
    g2.stage(stg);
    const size_t at_cp = stg.add(cp), at_vj = stg.add(&vj, sizeof(vj)), at_off = stg.add(off);
    upload(stg);
    const uint8_t* d = stage_.view<uint8_t>();
    tpoint_.as<uint32_t>(std::max(g1.terms, g2.terms) + 1);
    tscalar_.as<uint32_t>(std::max(g1.terms, g2.terms) + 1);
    stat_fme_ += (uint64_t)(g1.fme + 3 * g2.fme);
    run_msm<Fq>(ws1_, P.table.view<G1A>(), g1, d, nullptr, nullptr, arena, rec, err, tpoint_, tscalar_, st_);
    run_msm<Fq2>(ws2_, P.table2.view<G2A>(), g2, d, nullptr, nullptr, arena, rec, err + 1, tpoint_, tscalar_, st_);
    k_dv_copy<<<dim3(1, (unsigned)cp.size()), 32, 0, st>>>((uint32_t)cp.size(), reinterpret_cast<const CopyDesc*>(d + at_cp));
    DV_LAUNCH();
    run_verify(P, 1, 1, ANCHOR_TERMS, ANCHOR_EQS, reinterpret_cast<const VerifyJob*>(d + at_vj),
               reinterpret_cast<const uint64_t*>(d + at_off), verd, status);
    DV_CUDA(cudaMemcpyAsync(anc, an, ANCHOR_BYTES, cudaMemcpyDeviceToDevice, st));
    uint8_t* hout = pout_.as<uint8_t>(JOB_BYTES + 64 + ANCHOR_EQS);
    DV_CUDA(cudaMemcpyAsync(hout, rec, JOB_BYTES, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hout + JOB_BYTES, status, 4, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hout + JOB_BYTES + 8, err, 8, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hout + JOB_BYTES + 64, verd, ANCHOR_EQS, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    uint32_t hst, herr[2];
    memcpy(&hst, hout + JOB_BYTES, 4);
    memcpy(herr, hout + JOB_BYTES + 8, 8);
    if (herr[0] != 0xffffffffu || herr[1] != 0xffffffffu) throw CudaFailure("anchor MSM read a non-canonical scalar");
    bool ok = hst == 0;
    for (uint32_t e = 0; e < ANCHOR_EQS; ++e) ok &= hout[JOB_BYTES + 64 + e] == 1;
    job.ok = ok;
    job.anchor_bytes.assign(hout + RA, hout + RA + ANCHOR_BYTES);
    memcpy(job.public_h, hout + SIDE_PUBNEW, 64);
    if (!ok) job.error = hst & 4 ? "multiplication relation is not divisible by X^n - 1" : "proof failed verification";
}

// derive_h_sparse (dynamo.rs:462-476): h[i] += v, h[sigma(i)] -= v, zeros dropped.
std::map<uint32_t, hf::Fr> h_sparse(uint32_t n, const std::map<uint32_t, Canon>& entries) {
    std::map<uint32_t, hf::Fr> h;
    for (const auto& e : entries) {
        hf::Fr v;
        memcpy(v.v, e.second.data(), 32);  // canonical values: additions stay canonical
        auto& a = h[e.first];
        a = hf::add(a, v);
        auto& b = h[sigma_of(n, e.first)];
        b = hf::sub(b, v);
    }
    for (auto it = h.begin(); it != h.end();) it = hf::is_zero(it->second) ? h.erase(it) : std::next(it);
    return h;
}

// A batch of updates of sessions over the same parameters, in one set of
// launches: sparse proofs (prove_delta_sparse_traced, dynaverse/sparse.rs:
// 79-276, for every job at once) and re-anchors (the anchor of the new
// witness: the old anchor plus the delta's linear commitments, and a fresh
// multiplication quotient), each verified on the device before it is
// published (verify_delta_with_checks / verify_anchor_with_checks and the
// public-input identity, session.rs:126-131, dynaverse.rs:447).
void Engine::run_sparse(Params& P, std::vector<Job*>& jobs) {
    const uint32_t n = P.n, B = (uint32_t)jobs.size();
    const cudaStream_t st = st_;
    struct JL {
        bool rb = false;
        uint32_t d = 0, h = 0, pd = 0, a = 0;
        uint64_t E = 0, Hs = 0, FI = 0, PD = 0, FO = 0, DN = 0, R0 = 0;
        uint64_t LE = 0, LH = 0, LS[6] = {}, LSN[6] = {}, LA = 0, LPD = 0;
    };
    std::vector<JL> jl(B);
    std::vector<Canon> ain;
    std::vector<uint32_t> lrow, lsc;
    std::vector<std::pair<uint32_t, uint64_t>> scat;  // (job, arena source) for re-anchor rows; dst below
    std::vector<uint64_t> scat_rel;
    for (uint32_t j = 0; j < B; ++j) {
        Job& J = *jobs[j];
        Session& S = *J.S;
        JL& L = jl[j];
        L.rb = J.rebuild;
        L.d = (uint32_t)J.delta.size();
        L.E = ain.size();
        L.LE = lrow.size();
        uint32_t e = 0;
        for (const auto& kv : J.delta) {
            ain.push_back(kv.second);
            lrow.push_back(kv.first);
            lsc.push_back((uint32_t)(L.E + e));
            if (L.rb && kv.first >= 3 * n) {  // the delta of wires s4..s6 for the new coefficients
                scat.push_back({j, L.E + e});
                scat_rel.push_back((uint64_t)(kv.first / n - 3) * n + kv.first % n);
            }
            ++e;
        }
        const auto hm = h_sparse(n, J.delta);
        L.h = (uint32_t)hm.size();
        L.Hs = ain.size();
        L.LH = lrow.size();
        e = 0;
        for (const auto& kv : hm) {
            Canon c;
            memcpy(c.data(), kv.second.v, 32);
            ain.push_back(c);
            lrow.push_back(kv.first);
            lsc.push_back((uint32_t)(L.Hs + e++));
        }
        for (int t = 0; t < 6; ++t) {
            L.LS[t] = lrow.size();
            e = 0;
            for (const auto& kv : J.delta) {
                if (kv.first / n == (uint32_t)t) {
                    lrow.push_back(kv.first % n);
                    lsc.push_back((uint32_t)(L.E + e));
                }
                ++e;
            }
            L.LSN[t] = lrow.size() - L.LS[t];
        }
        std::set<uint32_t> aff;
        if (!L.rb)
            for (const auto& kv : J.delta)
                if (kv.first >= 3 * n) aff.insert(kv.first % n);
        L.a = (uint32_t)aff.size();
        L.FI = ain.size();
        for (int t = 0; t < 3; ++t)
            for (uint32_t i : aff) ain.push_back(anchor_value(S, (3 + t) * n + i));
        for (int t = 0; t < 3; ++t)
            for (uint32_t i : aff) {
                auto it = J.delta.find((3 + t) * n + i);
                ain.push_back(it == J.delta.end() ? Canon{0, 0, 0, 0} : it->second);
            }
        L.PD = ain.size();
        L.LPD = lrow.size();
        e = 0;
        for (const auto& kv : J.pedits) {
            hf::Fr nv, ov;
            memcpy(nv.v, kv.second.data(), 32);
            memcpy(ov.v, S.pub[kv.first].data(), 32);
            const hf::Fr d = hf::sub(nv, ov);
            if (hf::is_zero(d)) continue;
            Canon c;
            memcpy(c.data(), d.v, 32);
            ain.push_back(c);
            lrow.push_back((uint32_t)kv.first);
            lsc.push_back((uint32_t)(L.PD + e++));
        }
        L.pd = e;
        L.LA = lrow.size();
        for (uint32_t i : aff) {
            lrow.push_back(i);
            lsc.push_back(0);
        }
    }
    // arena outputs and scratch
    uint64_t top = ain.size(), scr = 0, amax = 0;
    std::vector<FieldJob> fj(B);
    std::vector<uint32_t> kjob(B + 1, 0);
    for (uint32_t j = 0; j < B; ++j) {
        JL& L = jl[j];
        L.FO = top;
        top += 19ull * L.a + 1;
        amax = std::max<uint64_t>(amax, L.a);
        kjob[j + 1] = kjob[j] + L.a;
    }
    for (uint32_t j = 0; j < B; ++j) {
        JL& L = jl[j];
        if (L.a) {
            L.DN = top;
            top += 4ull * n;
        }
        if (L.rb) {  // delta rows (3n), s4' padded (2n), s5' padded (2n), quotient (n)
            L.R0 = top;
            top += 8ull * n;
        }
        FieldJob& F = fj[j];
        F.a = L.a;
        F.aff = (uint32_t)L.LA;
        F.in = (uint32_t)L.FI;
        F.out = (uint32_t)L.FO;
        F.scr = (uint32_t)scr;
        scr += 22ull * L.a + 1;
        F.mat = (uint32_t)scr;
        scr += (uint64_t)L.a * L.a;
        F.dense = (uint32_t)L.DN;
        F.status = j;
        F.coef = jobs[j]->S->d_coef.view<Fr>();
    }
    if (top >= (1ull << 31) || scr >= (1ull << 31) || lrow.size() >= (1ull << 31))
        throw InvalidArgument("batch too large");
    std::vector<uint32_t> pairs;
    for (size_t k = 0; k < scat.size(); ++k) {
        pairs.push_back((uint32_t)(jl[scat[k].first].R0 + scat_rel[k]));
        pairs.push_back((uint32_t)scat[k].second);
    }
    // MSM launches: the linear fields (dynamo, wires, consistency, public
    // quotient, public differences); the affected-set fields and re-anchor
    // quotients; the G2 fields
    MsmBuild m1, m2, m3, md;  // md: the dense sets, over the c = 16 table
    std::vector<CopyDesc> cp, cp2;  // fixed fields: G1 on st_, G2 on st2_
    std::vector<VerifyJob> vj(B);
    std::vector<RebaseJob> rj;
    std::vector<uint64_t> off{0};
    uint8_t* out = out_.as<uint8_t>((uint64_t)B * JOB_BYTES);
    auto fo = [&](int f) { return P.fam_off[f]; };
    uint64_t terms = 0, fresh = 0;
    for (uint32_t j = 0; j < B; ++j) {
        const JL& L = jl[j];
        Session& S = *jobs[j]->S;
        const uint64_t rec = (uint64_t)j * JOB_BYTES;
        uint8_t* R = out + rec;
        const int dyf[5] = {F_ALPHA, F_BETA, F_H, F_Z, F_B};
        for (int k = 0; k < 5; ++k) {
            m1.seg(1, L.d, fo(dyf[k]), 0, L.LE);
            m1.end(rec + D_DYN + 64 * k);
        }
        m1.seg(1, L.d, fo(F_LX), 0, L.LE);
        m1.end(rec + D_DYN + 64 * DY_IZ);
        m1.seg(1, L.h, fo(F_LY), 0, L.LH);
        m1.end(rec + D_DYN + 64 * DY_IH);
        for (int t = 0; t < 6; ++t) {
            m1.seg(1, L.LSN[t], fo(F_LAG), 0, L.LS[t]);
            m1.end(rec + D_WIRES + 64 * t);
        }
        for (int t = 0; t < 6; ++t) {
            const uint64_t base = rec + D_CONS + 448 * t;
            m1.seg(1, L.d, fo(F_QAC0 + t), 0, L.LE);
            m1.end(base);
            const int cf[3] = {F_QCD, F_QBD, F_D};
            for (int k = 0; k < 3; ++k) {
                m1.seg(1, L.LSN[t], fo(cf[k]), 0, L.LS[t]);
                m1.end(base + 64 * (1 + k));
            }
            if (t == 0) {
                m1.seg(1, L.d, fo(F_ADEG), 0, L.LE);
                m1.end(base + 256);
            } else {
                cp.push_back({R + D_CONS + 448 * t + 256, R + D_CONS + 256, 64});
            }
            m1.seg(1, L.LSN[t], fo(F_BDEG), 0, L.LS[t]);
            m1.end(base + 320);
            m1.seg(1, L.LSN[t], fo(F_DDEG), 0, L.LS[t]);
            m1.end(base + 384);
        }
        m1.seg(1, L.d, fo(F_PQ), 0, L.LE);
        m1.end(rec + D_PZQ);
        m1.seg(1, L.pd, fo(F_PUBH), 0, L.LPD);
        m1.end(rec + SIDE_PDIFF);
        cp.push_back({R + D_W, R + D_DYN + 64 * DY_IZ, 64});
        cp.push_back({R + D_H, R + D_DYN + 64 * DY_IH, 64});
        if (L.rb) {
            // s5 of the delta (G2) and the new multiplication quotient
            m3.seg(1, L.LSN[4], P.fam2_off[F2_LAG], 0, L.LS[4]);
            m3.end(rec + D_AFF2);
            md.seg(0, n - 1, 0, L.R0 + 7ull * n, 0);
            md.end(rec + REC_ANCHOR + A_MQ);
            rj.push_back({R, S.d_anchor.view<uint8_t>()});
            vj[j] = VerifyJob{R, R + REC_ANCHOR, 0, (uint32_t)terms, (uint32_t)fresh, j};
            terms += ANCHOR_TERMS;
            fresh += 1;
            for (uint32_t c : eq_terms(false)) off.push_back(off.back() + c);
            continue;
        }
        // affected-set fields of a sparse proof
        const uint32_t a = L.a;
        const uint64_t FO = L.FO;
        m2.seg(0, a + 1, fo(F_KZG), FO + 0, 0);
        m2.end(rec + D_AFF1);
        if (a) {
            m2.seg(2, a, fo(F_LAG), FO + (a + 1), L.LA);
            m2.end(rec + D_UNAFF1);
        } else {
            cp.push_back({R + D_UNAFF1, P.consts.view<uint8_t>() + 64, 64});
            cp2.push_back({R + D_UNAFF2, P.consts.view<uint8_t>() + 128, 128});
        }
        for (int t = 0; t < 3; ++t) {
            m2.seg(0, a, fo(F_KZG), FO + 2 * a + 1 + t * a, 0);
            m2.end(rec + D_ALOC + 64 * t);
            m2.seg(0, a, fo(F_KZG), FO + 5 * a + 1 + t * a, 0);
            m2.end(rec + D_CLOC + 64 * t);
            m2.seg(2, a, fo(F_LAG), FO + 11 * a + 1 + t * a, L.LA);
            m2.seg(2, a, fo(F_OPENU), FO + 14 * a + 1 + t * a, L.LA);
            m2.end(rec + D_COPEN + 64 * t);
            m2.seg(0, a, fo(F_KZG), FO + 8 * a + 1 + t * a, 0);
            m2.end(rec + D_UZERO + 64 * t);
            if (a) {
                md.seg(0, n - a, 0, L.DN + (uint64_t)t * n, 0);
                md.end(rec + D_AOPEN + 64 * t);
            } else {
                cp.push_back({R + D_AOPEN + 64 * t, S.d_anchor.view<uint8_t>() + A_WIRES + 64 * (3 + t), 64});
            }
        }
        m2.seg(0, a ? a - 1 : 0, fo(F_KZG), FO + 18 * a + 1, 0);
        m2.end(rec + D_LQ);
        m3.seg(0, a + 1, P.fam2_off[F2_KZG], FO + 0, 0);
        m3.end(rec + D_AFF2);
        if (a) {
            m3.seg(2, a, P.fam2_off[F2_LAG], FO + (a + 1), L.LA);
            m3.end(rec + D_UNAFF2);
        }
        m3.seg(0, a, P.fam2_off[F2_KZG], FO + 17 * a + 1, 0);
        m3.end(rec + D_US5);
        vj[j] = VerifyJob{R, S.d_anchor.view<uint8_t>(), 1, (uint32_t)terms, (uint32_t)fresh, j};
        terms += DELTA_TERMS;
        fresh += 3;
        for (uint32_t c : eq_terms(true)) off.push_back(off.back() + c);
    }
    // the session's [public]_h goes to each record's input slot
    std::vector<uint8_t> pubh(64ull * B);
    for (uint32_t j = 0; j < B; ++j) memcpy(&pubh[64ull * j], jobs[j]->S->public_h, 64);
    Stager stg;
    m1.stage(stg);
    m2.stage(stg);
    m3.stage(stg);
    md.stage(stg);
    const size_t at_lrow = stg.add(lrow), at_lsc = stg.add(lsc), at_fj = stg.add(fj), at_kj = stg.add(kjob),
                 at_vj = stg.add(vj), at_off = stg.add(off), at_pub = stg.add(pubh), at_pairs = stg.add(pairs),
                 at_rj = stg.add(rj);
    upload(stg);
    const uint8_t* d = stage_.view<uint8_t>();
    std::vector<CopyDesc> cp0;
    for (uint32_t j = 0; j < B; ++j) cp0.push_back({out + (uint64_t)j * JOB_BYTES + SIDE_PUB, d + at_pub + 64ull * j, 64});
    Stager stg2;
    const size_t at_cp0 = stg2.add(cp0), at_cp = stg2.add(cp), at_cp2 = stg2.add(cp2);
    uint8_t* hs2 = pstage2_.as<uint8_t>(stg2.h.size());
    memcpy(hs2, stg2.h.data(), stg2.h.size());
    uint8_t* d2 = tmp_.as<uint8_t>(stg2.h.size());
    DV_CUDA(cudaMemcpyAsync(d2, hs2, stg2.h.size(), cudaMemcpyHostToDevice, st));

    Fr* arena = arena_.as<Fr>(std::max<uint64_t>(1, top));
    Fr* scratch = scr_.as<Fr>(std::max<uint64_t>(1, scr));
    uint32_t* status = status_.as<uint32_t>(B);
    const uint64_t eqs = off.size() - 1;
    // Every NTT batch of this pipeline is prepared before the first launch:
    // preparing synchronises the stream, which mid-pipeline would stall the
    // host behind the queued work and leave the GPU idle meanwhile.
    std::vector<std::pair<uint32_t, Fr*>> coefs;  // re-anchor jobs and their new coefficient buffers
    for (uint32_t j = 0; j < B; ++j)
        if (jl[j].rb) {
            take(jobs[j]->new_coef, 3ull * n * sizeof(Fr));
            take(jobs[j]->new_anchor, ANCHOR_BYTES);
            coefs.push_back({j, jobs[j]->new_coef.view<Fr>()});
        }
    const bool dense = kjob[B] > 0, rebuild = !coefs.empty();
    {
        std::vector<NttBatchItem> fwd, inv, r1, r2, r3;
        for (uint32_t j = 0; j < B; ++j) {
            if (!jl[j].a) continue;
            uint8_t* base = reinterpret_cast<uint8_t*>(arena + jl[j].DN);
            for (int r = 0; r < 4; ++r) fwd.push_back({base + 32ull * r * n, base + 32ull * r * n, (int)P.logn, NTT_COSET_FORWARD});
            for (int r = 0; r < 3; ++r) inv.push_back({base + 32ull * r * n, base + 32ull * r * n, (int)P.logn, NTT_COSET_INVERSE});
        }
        for (auto& jc : coefs) {
            uint8_t* base = reinterpret_cast<uint8_t*>(arena + jl[jc.first].R0);
            for (int t = 0; t < 3; ++t) r1.push_back({base + 32ull * t * n, base + 32ull * t * n, (int)P.logn, NTT_INVERSE});
            r2.push_back({base + 32ull * 3 * n, base + 32ull * 3 * n, (int)P.logn + 1, NTT_FORWARD});
            r2.push_back({base + 32ull * 5 * n, base + 32ull * 5 * n, (int)P.logn + 1, NTT_FORWARD});
            r3.push_back({base + 32ull * 3 * n, base + 32ull * 3 * n, (int)P.logn + 1, NTT_INVERSE});
        }
        if (dense) {
            ntt_batch_prepare(b_->ntt, nb_fwd_, fwd, st);
            ntt_batch_prepare(b_->ntt, nb_inv_, inv, st);
        }
        if (rebuild) {
            if (P.logn) ntt_batch_prepare(b_->ntt, nb_r1_, r1, st);  // a transform of one element is the identity
            ntt_batch_prepare(b_->ntt, nb_r2_, r2, st);
            ntt_batch_prepare(b_->ntt, nb_r3_, r3, st);
        }
    }
    uint8_t* verd = verdicts_.as<uint8_t>(std::max<uint64_t>(1, eqs));
    uint32_t* err = err_.as<uint32_t>(4);  // one word per MSM: m1, md, m3, m2
    if (!ain.empty()) {
        Canon* h = parena_.as<Canon>(ain.size());
        memcpy(h, ain.data(), 32 * ain.size());
        DV_CUDA(cudaMemcpyAsync(arena, h, 32 * ain.size(), cudaMemcpyHostToDevice, st));
    }
    const uint64_t e0 = now_ns();
    DV_CUDA(cudaMemsetAsync(out, 0, (uint64_t)B * JOB_BYTES, st));
    DV_CUDA(cudaMemsetAsync(status, 0, 4ull * B, st));
    DV_CUDA(cudaMemsetAsync(err, 0xff, 16, st));
    k_dv_copy<<<dim3(1, B), 32, 0, st>>>(B, reinterpret_cast<const CopyDesc*>(d2 + at_cp0));
    DV_LAUNCH();
    const uint32_t maxterms = md.terms + 1;
    tpoint_.as<uint32_t>(maxterms);
    tscalar_.as<uint32_t>(maxterms);
    tpoint3_.as<uint32_t>(std::max(m1.terms, m2.terms) + 1);  // m1 then m2 on st3_: sized once, before either
    tscalar3_.as<uint32_t>(std::max(m1.terms, m2.terms) + 1);
    const uint32_t* d_lrow = reinterpret_cast<const uint32_t*>(d + at_lrow);
    const uint32_t* d_lsc = reinterpret_cast<const uint32_t*>(d + at_lsc);
    stat_fme_ += (uint64_t)(m1.fme + m2.fme + md.fme + 3 * m3.fme);
    // m1 on st3_ once the inputs and the zeroed records are in place
    DV_CUDA(cudaEventRecord(ev_start_, st));
    DV_CUDA(cudaStreamWaitEvent(st3_, ev_start_, 0));
    run_msm<Fq>(ws3_, P.table.view<G1A>(), m1, d, d_lrow, d_lsc, arena, out, err, tpoint3_, tscalar3_, st3_);
    // field work of the affected sets
    FieldCtx c{reinterpret_cast<const FieldJob*>(d + at_fj), reinterpret_cast<const uint32_t*>(d + at_kj), B, d_lrow,
               P.wpow.view<Fr>(), P.inv1m.view<Fr>(), n, Fr{}, Fr{}, arena, scratch, status};
    memcpy(&c.n_m, P.n_m.v, 32);
    memcpy(&c.ninv_m, P.ninv_m.v, 32);
    const uint32_t K = kjob[B];
    if (!quot_smem_) {
        DV_CUDA(cudaFuncSetAttribute(k_dv_quot, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        quot_smem_ = true;
    }
    if (K) {
        k_dv_geom<<<(unsigned)((32ull * K + 127) / 128), 128, 0, st>>>(c);
        DV_LAUNCH();
    }
    uint64_t vanish_n = 1;  // the largest transform of k_dv_vanish
    while (vanish_n < amax + 1) vanish_n <<= 1;
    k_dv_vanish<<<B, 1024, vanish_n * sizeof(Fr), st>>>(c);
    DV_LAUNCH();
    if (K) {
        k_dv_lagmat<<<(unsigned)((32ull * K + 127) / 128), 128, 0, st>>>(c);
        DV_LAUNCH();
        k_dv_rows<<<(unsigned)((32ull * 13 * K + 127) / 128), 128, 0, st>>>(c);
        DV_LAUNCH();
        k_dv_combine<<<(K + 127) / 128, 128, 0, st>>>(c);
        DV_LAUNCH();
        k_dv_quot<<<B, 256, std::max<uint64_t>(1, 4 * amax) * sizeof(Fr), st>>>(c);
        DV_LAUNCH();
    }
    // The G2 side on st2_, once the field rows it reads exist: the G2 MSM,
    // the re-anchors' G2 field, the fresh G2 points and their pairing lines.
    // It overlaps the dense G1 work below, which touches none of its inputs.
    G2A* q = g2q_.as<G2A>(V_COUNT + fresh);
    lines_.as<uint8_t>((V_COUNT + fresh) * pairing_prepared_bytes());
    qinf_.as<uint32_t>(V_COUNT + fresh);
    tpoint2_.as<uint32_t>(m3.terms + 1);
    tscalar2_.as<uint32_t>(m3.terms + 1);
    DV_CUDA(cudaEventRecord(ev_fields_, st));
    DV_CUDA(cudaStreamWaitEvent(st2_, ev_fields_, 0));
    // m2 on st3_ after m1, once the field rows it reads exist
    DV_CUDA(cudaStreamWaitEvent(st3_, ev_fields_, 0));
    run_msm<Fq>(ws3_, P.table.view<G1A>(), m2, d, d_lrow, d_lsc, arena, out, err + 3, tpoint3_, tscalar3_, st3_);
    DV_CUDA(cudaEventRecord(ev_m1_, st3_));
    run_msm<Fq2>(ws2_, P.table2.view<G2A>(), m3, d, d_lrow, d_lsc, arena, out, err + 2, tpoint2_, tscalar2_, st2_);
    if (!cp2.empty()) {
        k_dv_copy<<<dim3(1, (unsigned)cp2.size()), 32, 0, st2_>>>((uint32_t)cp2.size(),
                                                                  reinterpret_cast<const CopyDesc*>(d2 + at_cp2));
        DV_LAUNCH();
    }
    if (!rj.empty()) {
        k_dv_rebase<<<(unsigned)((rj.size() + 63) / 64), 64, 0, st2_>>>(reinterpret_cast<const RebaseJob*>(d + at_rj),
                                                                    (uint32_t)rj.size(), REBASE_FIELDS - 1,
                                                                    REBASE_FIELDS);
        DV_LAUNCH();
    }
    k_dv_fresh<<<(B + 31) / 32, 32, 0, st2_>>>(reinterpret_cast<const VerifyJob*>(d + at_vj), B, q);
    DV_LAUNCH();
    prepare_lines(P, q, fresh, st2_);
    DV_CUDA(cudaEventRecord(ev_g2_, st2_));
    if (K) {
        // anchor openings: (s_t - r_t) / A on the coset 5 H
        const uint64_t t4 = 4ull * n * B;
        k_dv_numer<<<(unsigned)((t4 + 255) / 256), 256, 0, st>>>(c);
        DV_LAUNCH();
        ntt_batch_enqueue(nb_fwd_, st);
        k_dv_divq<<<(unsigned)(((uint64_t)((n + DQ - 1) / DQ) * B + 127) / 128), 128, 0, st>>>(c);
        DV_LAUNCH();
        ntt_batch_enqueue(nb_inv_, st);
        k_dv_degcheck<<<(unsigned)((3ull * n * B + 255) / 256), 256, 0, st>>>(c);
        DV_LAUNCH();
    }
    // re-anchors: new coefficients s_t + delta_t, then (s4 s5 - s6) / (X^n - 1)
    if (rebuild) {
        for (auto& jc : coefs)
            DV_CUDA(cudaMemsetAsync(arena + jl[jc.first].R0, 0, 32ull * 3 * n, st));
        if (!scat.empty()) {
            k_dv_scatter<<<(unsigned)((scat.size() + 255) / 256), 256, 0, st>>>(
                reinterpret_cast<const uint32_t*>(d + at_pairs), (uint32_t)scat.size(), arena);
            DV_LAUNCH();
        }
        if (P.logn) ntt_batch_enqueue(nb_r1_, st);
        const unsigned g3 = (unsigned)((3ull * n + 255) / 256), g2n = (unsigned)((2ull * n + 255) / 256);
        for (auto& jc : coefs) {
            Fr* rows = arena + jl[jc.first].R0;
            k_dv_vadd<<<g3, 256, 0, st>>>(jc.second, jobs[jc.first]->S->d_coef.view<Fr>(), rows, 3ull * n);
            DV_LAUNCH();
            k_dv_pad<<<g2n, 256, 0, st>>>(jc.second, n, rows + 3ull * n, 2ull * n);
            DV_LAUNCH();
            k_dv_pad<<<g2n, 256, 0, st>>>(jc.second + n, n, rows + 5ull * n, 2ull * n);
            DV_LAUNCH();
        }
        ntt_batch_enqueue(nb_r2_, st);
        for (auto& jc : coefs) {
            Fr* rows = arena + jl[jc.first].R0;
            k_dv_pmul<<<g2n, 256, 0, st>>>(rows + 3ull * n, rows + 5ull * n, 2ull * n);
            DV_LAUNCH();
        }
        ntt_batch_enqueue(nb_r3_, st);
        for (auto& jc : coefs) {
            Fr* rows = arena + jl[jc.first].R0;
            k_dv_mq<<<(n + 255) / 256, 256, 0, st>>>(rows + 3ull * n, jc.second + 2ull * n, n, rows + 7ull * n,
                                                     status + jc.first);
            DV_LAUNCH();
        }
    }
    run_msm<Fq>(ws1_, P.table_dense.view<G1A>(), md, d, d_lrow, d_lsc, arena, out, err + 1, tpoint_, tscalar_, st, TCD,
                TWD);
    // the record copies, the re-anchors' G1 fields and the verification
    // terms read m1's and m2's outputs
    DV_CUDA(cudaStreamWaitEvent(st, ev_m1_, 0));
    if (!cp.empty()) {
        k_dv_copy<<<dim3(1, (unsigned)cp.size()), 32, 0, st>>>((uint32_t)cp.size(), reinterpret_cast<const CopyDesc*>(d2 + at_cp));
        DV_LAUNCH();
    }
    if (!rj.empty()) {
        const uint32_t tot = (uint32_t)rj.size() * (REBASE_FIELDS - 1);
        k_dv_rebase<<<(tot + 63) / 64, 64, 0, st>>>(reinterpret_cast<const RebaseJob*>(d + at_rj), (uint32_t)rj.size(),
                                                    0, REBASE_FIELDS - 1);
        DV_LAUNCH();
    }
    // verification: the G1 terms here, then the pairings once st2_ is done
    G1A* tp1 = terms_p_.as<G1A>(std::max<uint64_t>(1, terms));
    uint32_t* tq1 = terms_q_.as<uint32_t>(std::max<uint64_t>(1, terms));
    k_dv_terms<<<dim3(B, TERM_PIECES), 32, 0, st>>>(reinterpret_cast<const VerifyJob*>(d + at_vj), B, host_g1(P.g1), host_g1(P.mvg1),
                                 tp1, tq1, status);
    DV_LAUNCH();
    DV_CUDA(cudaStreamWaitEvent(st, ev_g2_, 0));
    pairing_check_prepared(*b_, tp1, terms, lines_.view<uint8_t>(), qinf_.view<uint32_t>(), tq1,
                           reinterpret_cast<const uint64_t*>(d + at_off), eqs, verd, st);
    for (auto& jc : coefs) {
        uint8_t* an = jobs[jc.first]->new_anchor.view<uint8_t>();
        DV_CUDA(cudaMemcpyAsync(an, out + (uint64_t)jc.first * JOB_BYTES + REC_ANCHOR, ANCHOR_BYTES,
                                cudaMemcpyDeviceToDevice, st));
    }
    const uint64_t ob = (uint64_t)B * JOB_BYTES;
    uint8_t* hout = pout_.as<uint8_t>(ob + 4ull * B + 16 + eqs);
    DV_CUDA(cudaMemcpyAsync(hout, out, ob, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hout + ob, status, 4ull * B, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hout + ob + 4ull * B, err, 16, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hout + ob + 4ull * B + 16, verd, eqs, cudaMemcpyDeviceToHost, st));
    const uint64_t w0 = now_ns();
    stat_enqueue_ns_ += w0 - e0;
    DV_CUDA(cudaStreamSynchronize(st));
    stat_wait_ns_ += now_ns() - w0;
    if (md.terms) {
        float ms = 0;
        DV_CUDA(cudaEventElapsedTime(&ms, ws1_.timeline.acc_ev[0], ws1_.timeline.acc_ev[1]));
        stat_dense_ns_ += (uint64_t)(ms * 1e6);
        stat_dense_adds_ += (uint64_t)md.terms * TWD;
    }
    if (dense) {
        ntt_batch_check(nb_fwd_, st);
        ntt_batch_check(nb_inv_, st);
    }
    if (rebuild) {
        if (P.logn) ntt_batch_check(nb_r1_, st);
        ntt_batch_check(nb_r2_, st);
        ntt_batch_check(nb_r3_, st);
    }
    uint32_t herr[4];
    memcpy(herr, hout + ob + 4ull * B, 16);
    for (int i = 0; i < 4; ++i)
        if (herr[i] != 0xffffffffu) throw CudaFailure("update MSM read a non-canonical scalar");
    for (uint32_t j = 0; j < B; ++j) {
        Job& J = *jobs[j];
        uint32_t hst;
        memcpy(&hst, hout + ob + 4ull * j, 4);
        const bool ok = hst == 0;
        const uint8_t* r = hout + (uint64_t)j * JOB_BYTES;
        J.proof.assign(PROOF_BYTES, 0);
        if (J.rebuild) {
            J.anchor_bytes.assign(r + REC_ANCHOR, r + REC_ANCHOR + ANCHOR_BYTES);
            memcpy(J.proof.data(), r + REC_ANCHOR, ANCHOR_BYTES);
            const uint64_t tail[3] = {0, J.generation, J.generation};
            memcpy(J.proof.data() + ANCHOR_BYTES + DELTA_BYTES, tail, 24);
        } else {
            memcpy(J.proof.data(), J.S->anchor_bytes.data(), ANCHOR_BYTES);
            memcpy(J.proof.data() + ANCHOR_BYTES, r, DELTA_BYTES);
            const uint64_t tail[3] = {1, J.S->anchor_generation, J.generation};
            memcpy(J.proof.data() + ANCHOR_BYTES + DELTA_BYTES, tail, 24);
        }
        memcpy(J.public_h, r + SIDE_PUBNEW, 64);
        J.ok = ok;
        J.error = hst & 1   ? "polynomial division has a nonzero remainder"
                  : hst & 2 ? "anchor opening division has a nonzero remainder"
                  : hst & 4 ? "multiplication relation is not divisible by X^n - 1"
                            : (J.rebuild ? "updated proof failed public verification"
                                         : "sparse session proof failed verification");
    }
    // verdicts: each job's equations are a contiguous range of `off`
    uint64_t eq = 0;
    for (uint32_t j = 0; j < B; ++j) {
        const uint64_t cnt = jl[j].rb ? ANCHOR_EQS : DELTA_EQS;
        const uint8_t* v = hout + ob + 4ull * B + 16 + eq;
        for (uint64_t e = 0; e < cnt; ++e) jobs[j]->ok &= v[e] == 1;
        eq += cnt;
    }
}

// ================================================================ sessions
void read_canon(const uint8_t* b, uint64_t count, std::vector<Canon>& out, const char* what) {
    out.resize(count);
    for (uint64_t i = 0; i < count; ++i) {
        if (!canon_ok(b + 32 * i)) throw InvalidArgument(std::string("non-canonical ") + what + " value");
        memcpy(out[i].data(), b + 32 * i, 32);
    }
}

// ToyCircuit::validate on the given gates (toy_circuit.rs:72-90).
template <class Wire, class Input>
void check_gates(uint64_t n, const std::vector<uint64_t>& gates, Wire wire, Input input) {
    for (uint64_t i : gates) {
        if (wire(i) != input(i)) throw InvalidArgument("public copy constraint fails at " + std::to_string(i));
        if (wire(2 * n + i) != wire(3 * n + i))
            throw InvalidArgument("wire copy constraint fails at " + std::to_string(i));
        const hf::Fr s = hf::add(as_fr(wire(i)), as_fr(wire(n + i)));  // canonical operands: canonical sum
        if (!hf::eq(s, as_fr(wire(2 * n + i)))) throw InvalidArgument("addition gate fails at " + std::to_string(i));
        const hf::Fr prod = hf::mul(mont_of(wire(3 * n + i)), mont_of(wire(4 * n + i)));
        if (!hf::eq(prod, mont_of(wire(5 * n + i))))
            throw InvalidArgument("multiplication gate fails at " + std::to_string(i));
    }
}

uint64_t Engine::open_impl(uint64_t pid, const uint8_t* pubb, const uint8_t* witb, uint8_t* proof) {
    Params* P = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = params_.find(pid);
        if (it == params_.end()) throw InvalidArgument("unknown parameters");
        P = it->second.get();
    }
    const uint64_t n = P->n;
    std::vector<Canon> pub, w;
    read_canon(pubb, n, pub, "public input");
    read_canon(witb, 6 * n, w, "witness");
    std::vector<uint64_t> all(n);
    for (uint64_t i = 0; i < n; ++i) all[i] = i;
    check_gates(n, all, [&](uint64_t i) { return w[i]; }, [&](uint64_t i) { return pub[i]; });
    const uint64_t footprint = 3 * n * 32 + ANCHOR_BYTES + 256;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (resident_ + footprint > budget_)
            throw InvalidArgument("session does not fit the HBM budget (" + std::to_string(resident_) + " + " +
                                  std::to_string(footprint) + " > " + std::to_string(budget_) + " bytes)");
    }
    Job job;
    run_anchor(*P, w, pub, job);
    if (!job.ok) throw InvalidArgument("initial session proof failed verification (" + job.error + ")");
    auto S = std::make_unique<Session>();
    S->P = P;
    S->n = (uint32_t)n;
    S->pub = std::move(pub);
    S->current = std::move(w);
    S->anchor_bytes = job.anchor_bytes;
    std::swap(S->d_anchor.ptr, job.new_anchor.ptr);
    std::swap(S->d_anchor.cap, job.new_anchor.cap);
    std::swap(S->d_coef.ptr, job.new_coef.ptr);
    std::swap(S->d_coef.cap, job.new_coef.cap);
    memcpy(S->public_h, job.public_h, 64);
    S->proof.assign(PROOF_BYTES, 0);
    memcpy(S->proof.data(), job.anchor_bytes.data(), ANCHOR_BYTES);
    S->footprint = footprint;
    memcpy(proof, S->proof.data(), PROOF_BYTES);
    std::lock_guard<std::mutex> lk(mu_);
    S->id = next_id_++;
    resident_ += footprint;
    const uint64_t id = S->id;
    sessions_[id] = std::move(S);
    return id;
}

// DynaverseVerifyingKey::verify (dynaverse.rs:978-1016) of proof bytes on
// the device: the anchor's equations (with the public-input identity when
// there is no delta), the delta's, and the identity
// anchor h + delta h + [public]_h == 0.
bool Engine::verify_impl(uint64_t pid, const uint8_t* pubb, const uint8_t* proof) {
    Params* P = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = params_.find(pid);
        if (it == params_.end()) throw InvalidArgument("unknown parameters");
        P = it->second.get();
    }
    const uint64_t n = P->n;
    std::vector<Canon> pub;
    read_canon(pubb, n, pub, "public input");
    uint64_t tail[3];
    memcpy(tail, proof + ANCHOR_BYTES + DELTA_BYTES, 24);
    const bool has = tail[0] != 0;
    if (tail[0] > 1 || tail[1] > tail[2] || has != (tail[1] < tail[2])) return false;
    // points must deserialise: canonical coordinates on their curves
    const cudaStream_t st = st_;
    uint8_t* out = out_.as<uint8_t>(2 * JOB_BYTES);
    DV_CUDA(cudaMemsetAsync(out, 0, 2 * JOB_BYTES, st));
    DV_CUDA(cudaMemcpyAsync(out + REC_ANCHOR, proof, ANCHOR_BYTES, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(out + JOB_BYTES, proof + ANCHOR_BYTES, DELTA_BYTES, cudaMemcpyHostToDevice, st));
    // every G1 / G2 field must parse (codec.rs:25-111): checked by converting
    // them all; the G2 fields of the layout are known
    static const std::vector<uint64_t> g2a = {A_S5G2}, g2d = {D_AFF2, D_UNAFF2, D_US5};
    std::vector<uint8_t> g1w, g2w;
    auto collect = [&](const uint8_t* base, uint64_t len, const std::vector<uint64_t>& g2off) {
        for (uint64_t o = 0; o < len;) {
            if (std::find(g2off.begin(), g2off.end(), o) != g2off.end()) {
                g2w.insert(g2w.end(), base + o, base + o + 128);
                o += 128;
            } else {
                g1w.insert(g1w.end(), base + o, base + o + 64);
                o += 64;
            }
        }
    };
    collect(proof, ANCHOR_BYTES, g2a);
    if (has) collect(proof + ANCHOR_BYTES, DELTA_BYTES, g2d);
    uint8_t* d_g1 = arena_.as<uint8_t>(g1w.size() + g2w.size() + 32 * n);
    uint8_t* d_g2 = d_g1 + g1w.size();
    Fr* d_pub = reinterpret_cast<Fr*>(d_g2 + g2w.size());
    DV_CUDA(cudaMemcpyAsync(d_g1, g1w.data(), g1w.size(), cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(d_g2, g2w.data(), g2w.size(), cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(d_pub, pub.data(), 32 * n, cudaMemcpyHostToDevice, st));
    uint32_t* bad = err_.as<uint32_t>(4);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, 16, st));
    convert_points<Fq>(d_g1, terms_p_.as<G1A>(g1w.size() / 64), g1w.size() / 64, bad, st);
    convert_points<Fq2>(d_g2, g2q_.as<G2A>(g2w.size() / 128), g2w.size() / 128, bad + 1, st);
    uint32_t hb[2];
    DV_CUDA(cudaMemcpyAsync(hb, bad, 8, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (hb[0] != 0xffffffffu || hb[1] != 0xffffffffu) return false;
    // [public]_h
    MsmBuild mb;
    mb.seg(0, n, P->fam_off[F_PUBH], 0, 0);
    mb.end(has ? JOB_BYTES + SIDE_PDIFF : SIDE_PDIFF);
    std::vector<VerifyJob> vj;
    vj.push_back(VerifyJob{out, out + REC_ANCHOR, has ? 2u : 0u, 0, 0, 0});
    if (has) vj.push_back(VerifyJob{out + JOB_BYTES, out + REC_ANCHOR, 1, ANCHOR_TERMS, 1, 1});
    std::vector<uint64_t> off = eq_offsets(1, false);
    if (has) {
        const std::vector<uint64_t> d2 = eq_offsets(1, true);
        for (size_t i = 1; i < d2.size(); ++i) off.push_back(off[ANCHOR_EQS] + d2[i]);
    }
    Stager stg;
    mb.stage(stg);
    const size_t at_vj = stg.add(vj), at_off = stg.add(off);
    upload(stg);
    const uint8_t* d = stage_.view<uint8_t>();
    uint32_t* status = status_.as<uint32_t>(2);
    uint32_t* err = err_.as<uint32_t>(1);
    DV_CUDA(cudaMemsetAsync(status, 0, 8, st));
    DV_CUDA(cudaMemsetAsync(err, 0xff, 4, st));
    tpoint_.as<uint32_t>(n + 1);
    tscalar_.as<uint32_t>(n + 1);
    run_msm<Fq>(ws1_, P->table.view<G1A>(), mb, d, nullptr, nullptr, d_pub, out, err, tpoint_, tscalar_, st_);
    const uint64_t eqs = off.size() - 1;
    uint8_t* verd = verdicts_.as<uint8_t>(eqs);
    run_verify(*P, (uint32_t)vj.size(), has ? 4 : 1, off.back(), eqs, reinterpret_cast<const VerifyJob*>(d + at_vj),
               reinterpret_cast<const uint64_t*>(d + at_off), verd, status);
    std::vector<uint8_t> hv(eqs + 8);
    DV_CUDA(cudaMemcpyAsync(hv.data(), verd, eqs, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaMemcpyAsync(hv.data() + eqs, status, 8, cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    uint32_t hs[2];
    memcpy(hs, hv.data() + eqs, 8);
    if (hs[0] || hs[1]) return false;
    for (uint64_t e = 0; e < eqs; ++e)
        if (hv[e] != 1) return false;
    return true;
}

// UpdateSession::apply's host bookkeeping (session.rs:53-109): canonical
// edits, no-op detection, gate checks on the dirty gates, the new anchor
// differences, and the choice between a sparse proof and a re-anchor.
void Engine::stage_job(Request& r, Session* S, Job& job) {
    job.req = &r;
    job.S = S;
    const uint64_t n = S->n;
    for (size_t k = 0; k < r.idx.size(); ++k) job.edits[r.idx[k]] = r.vals[k];  // later entries win
    for (size_t k = 0; k < r.pidx.size(); ++k) job.pedits[r.pidx[k]] = r.pvals[k];
    if (!job.edits.empty() && job.edits.rbegin()->first >= 6 * n)
        throw InvalidArgument("update index " + std::to_string(job.edits.rbegin()->first) +
                              " out of range (witness len " + std::to_string(6 * n) + ")");
    if (!job.pedits.empty() && job.pedits.rbegin()->first >= n)
        throw InvalidArgument("update index " + std::to_string(job.pedits.rbegin()->first) +
                              " out of range (witness len " + std::to_string(n) + ")");
    std::set<uint64_t> dirty;
    bool changed = false;
    for (const auto& e : job.edits)
        if (e.second != S->current[e.first]) {
            changed = true;
            dirty.insert(e.first % n);
        }
    for (const auto& e : job.pedits)
        if (e.second != S->pub[e.first]) {
            changed = true;
            dirty.insert(e.first);
        }
    if (!changed) return;  // generation 0: the caller returns the current proof
    auto wire = [&](uint64_t i) {
        auto it = job.edits.find(i);
        return it != job.edits.end() ? it->second : S->current[i];
    };
    auto input = [&](uint64_t i) {
        auto it = job.pedits.find(i);
        return it != job.pedits.end() ? it->second : S->pub[i];
    };
    check_gates(n, std::vector<uint64_t>(dirty.begin(), dirty.end()), wire, input);
    job.generation = S->generation + 1;
    job.delta = S->delta;
    for (const auto& e : job.edits) {
        const hf::Fr diff = hf::sub(as_fr(e.second), as_fr(anchor_value(*S, e.first)));
        if (hf::is_zero(diff)) job.delta.erase((uint32_t)e.first);
        else {
            Canon c;
            memcpy(c.data(), diff.v, 32);
            job.delta[(uint32_t)e.first] = c;
        }
    }
    // A re-anchor proves the updated witness from scratch (session.rs:92).
    // Every gate of it holds: the session's witness satisfied the circuit
    // (checked in full when the session opened) and this update's dirty
    // gates were checked above, so no full pass is repeated here.
    if (job.delta.size() >= S->P->rebuild_interval) job.rebuild = true;
}

void Engine::process(std::vector<Request>& batch, std::vector<Session*>& sess, std::vector<Outcome>& outs) {
    std::vector<Job> jobs(batch.size());
    std::map<Params*, std::vector<Job*>> groups;
    std::vector<bool> active(batch.size(), false);
    for (size_t r = 0; r < batch.size(); ++r) {
        if (!sess[r]) {
            outs[r].status = -1;
            outs[r].error = "unknown session";
            continue;
        }
        try {
            stage_job(batch[r], sess[r], jobs[r]);
        } catch (const InvalidArgument& e) {
            outs[r].status = -1;
            outs[r].error = e.what();
            continue;
        }
        if (!jobs[r].generation) {  // no-op (session.rs:69)
            outs[r].proof = sess[r]->proof;
            continue;
        }
        active[r] = true;
        groups[sess[r]->P].push_back(&jobs[r]);  // sparse proofs and re-anchors share the batch
    }
    try {
        for (auto& g : groups) run_sparse(*g.first, g.second);
    } catch (const InvalidArgument& e) {
        for (size_t r = 0; r < batch.size(); ++r)
            if (active[r]) {
                outs[r].status = -1;
                outs[r].error = e.what();
                active[r] = false;
            }
    } catch (const std::exception& e) {
        for (size_t r = 0; r < batch.size(); ++r)
            if (active[r]) {
                outs[r].status = -2;
                outs[r].error = e.what();
                active[r] = false;
            }
    }
    if (std::any_of(outs.begin(), outs.end(), [](const Outcome& o) { return o.status != 0; })) {
        // a batch that stopped part way may have left work queued on the three
        // streams: let it finish before the next batch reuses the buffers (the
        // statuses are ignored; a lost context shows in the next batch's calls)
        for (cudaStream_t q : {st_, st2_, st3_})
            if (q) cudaStreamSynchronize(q);
        cudaGetLastError();
    }
    // publish (session.rs:132-141): only proofs that verified change state
    std::lock_guard<std::mutex> lk(mu_);
    for (size_t r = 0; r < batch.size(); ++r) {
        if (!active[r]) continue;
        Job& J = jobs[r];
        Session& S = *J.S;
        if (!J.ok) {
            outs[r].status = -1;
            outs[r].error = J.error;
            continue;
        }
        for (const auto& e : J.edits) S.current[e.first] = e.second;
        for (const auto& e : J.pedits) S.pub[e.first] = e.second;
        if (J.rebuild) {
            S.delta.clear();
            S.anchor_generation = J.generation;
            S.anchor_bytes = J.anchor_bytes;
            std::swap(S.d_anchor.ptr, J.new_anchor.ptr);
            std::swap(S.d_anchor.cap, J.new_anchor.cap);
            std::swap(S.d_coef.ptr, J.new_coef.ptr);
            std::swap(S.d_coef.cap, J.new_coef.cap);
            J.proof.assign(PROOF_BYTES, 0);
            memcpy(J.proof.data(), J.anchor_bytes.data(), ANCHOR_BYTES);
            const uint64_t tail[3] = {0, J.generation, J.generation};
            memcpy(J.proof.data() + ANCHOR_BYTES + DELTA_BYTES, tail, 24);
            stat_rebuilds_++;
        } else {
            S.delta = std::move(J.delta);
            stat_sparse_++;
        }
        S.generation = J.generation;
        S.proof = J.proof;
        memcpy(S.public_h, J.public_h, 64);
        outs[r].proof = J.proof;
        outs[r].res.rebuilt = J.rebuild ? 1 : 0;
    }
    // the buffers a re-anchor swapped out of its session (or did not use)
    for (auto& J : jobs) {
        give(J.new_coef);
        give(J.new_anchor);
    }
}

int fail_text(int status, const std::string& msg, char* error, size_t cap) {
    if (error && cap) {
        const size_t k = std::min(cap - 1, msg.size());
        memcpy(error, msg.data(), k);
        error[k] = '\0';
    }
    return status;
}

template <class Fn>
int dv_guard(char* error, size_t cap, Fn&& fn) {
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

using dv::Engine;

extern "C" int dvgpu_dynaverse_create(uint64_t hbm_budget_bytes, uint32_t max_batch, void** engine, char* error,
                                      size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine) throw dv::InvalidArgument("null engine output");
        *engine = nullptr;
        *engine = new Engine(hbm_budget_bytes, max_batch);
    });
}

extern "C" void dvgpu_dynaverse_destroy(void* engine) { delete static_cast<Engine*>(engine); }

extern "C" int dvgpu_dynaverse_params_create(void* engine, size_t n, const uint8_t* tau_x, const uint8_t* tau_y,
                                             uint64_t* params, char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine || !tau_x || !tau_y || !params) throw dv::InvalidArgument("invalid parameter arguments");
        *params = static_cast<Engine*>(engine)->params_create(n, tau_x, tau_y);
    });
}

extern "C" int dvgpu_dynaverse_params_destroy(void* engine, uint64_t params, char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine) throw dv::InvalidArgument("null engine");
        static_cast<Engine*>(engine)->params_destroy(params);
    });
}

extern "C" int dvgpu_dynaverse_params_info(void* engine, uint64_t params, DvgpuDynaverseParamsInfo* info,
                                           char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine || !info) throw dv::InvalidArgument("invalid arguments");
        static_cast<Engine*>(engine)->params_info(params, info);
    });
}

extern "C" int dvgpu_dynaverse_session_open(void* engine, uint64_t params, const uint8_t* public_inputs,
                                            const uint8_t* witness, uint64_t* session, uint8_t* proof, char* error,
                                            size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine || !public_inputs || !witness || !session || !proof)
            throw dv::InvalidArgument("invalid session arguments");
        *session = static_cast<Engine*>(engine)->open_session(params, public_inputs, witness, proof);
    });
}

extern "C" int dvgpu_dynaverse_session_close(void* engine, uint64_t session, char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine) throw dv::InvalidArgument("null engine");
        static_cast<Engine*>(engine)->close_session(session);
    });
}

extern "C" int dvgpu_dynaverse_session_state(void* engine, uint64_t session, uint8_t* witness,
                                             uint8_t* public_inputs, uint8_t* proof, uint64_t* anchor_distance,
                                             char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine) throw dv::InvalidArgument("null engine");
        static_cast<Engine*>(engine)->session_state(session, witness, public_inputs, proof, anchor_distance);
    });
}

extern "C" int dvgpu_dynaverse_submit(void* engine, uint64_t session, const uint64_t* indices, const uint8_t* values,
                                      size_t count, const uint64_t* public_indices, const uint8_t* public_values,
                                      size_t public_count, uint64_t* ticket, char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine || !ticket || (count && (!indices || !values)) ||
            (public_count && (!public_indices || !public_values)))
            throw dv::InvalidArgument("invalid update arguments");
        *ticket = static_cast<Engine*>(engine)->submit(session, indices, values, count, public_indices,
                                                       public_values, public_count);
    });
}

extern "C" int dvgpu_dynaverse_wait(void* engine, uint64_t ticket, uint8_t* proof, DvgpuDynaverseResult* result,
                                    char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine) throw dv::InvalidArgument("null engine");
        static_cast<Engine*>(engine)->wait(ticket, proof, result);
    });
}

extern "C" int dvgpu_dynaverse_update(void* engine, uint64_t session, const uint64_t* indices, const uint8_t* values,
                                      size_t count, const uint64_t* public_indices, const uint8_t* public_values,
                                      size_t public_count, uint8_t* proof, char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine || !proof || (count && (!indices || !values)) ||
            (public_count && (!public_indices || !public_values)))
            throw dv::InvalidArgument("invalid update arguments");
        Engine* e = static_cast<Engine*>(engine);
        const uint64_t t = e->submit(session, indices, values, count, public_indices, public_values, public_count);
        e->wait(t, proof, nullptr);
    });
}

extern "C" int dvgpu_dynaverse_verify(void* engine, uint64_t params, const uint8_t* public_inputs,
                                      const uint8_t* proof, uint8_t* accepted, char* error, size_t cap) {
    return dv::dv_guard(error, cap, [&] {
        if (!engine || !public_inputs || !proof || !accepted) throw dv::InvalidArgument("invalid verify arguments");
        static_cast<Engine*>(engine)->verify(params, public_inputs, proof, accepted);
    });
}

extern "C" int dvgpu_dynaverse_set_max_batch(void* engine, uint32_t max_batch) {
    if (!engine) return -1;
    static_cast<Engine*>(engine)->set_max_batch(max_batch);
    return 0;
}

extern "C" int dvgpu_dynaverse_stats(void* engine, DvgpuDynaverseStats* out) {
    if (!engine || !out) return -1;
    *out = static_cast<Engine*>(engine)->stats();
    return 0;
}
