// Device polynomial toolkit over BN254 Fr: products, exact division and the
// subproduct-tree operations of the sparse update
// (crates/protocol/src/domain/fast.rs: SubproductTree :11-139,
// newton_divide_exact_with_backend :236-240, fft_multiply_with_backend
// :213-234; callers crates/protocol/src/dynaverse/sparse.rs:125-236).
//
// Every output is fixed by exact arithmetic -- a field element, or a
// coefficient vector trimmed as domain.rs:339-346 (no trailing zeros, at
// least one entry) -- so the device reaches the same values by the route
// that suits the GPU:
//
//  * product: forward NTTs of both operands padded to N = next_pow2(l+r-1),
//    pointwise product, inverse NTT (the reference's own route);
//  * exact division a / b: forward NTTs of a and b on a coset sH with
//    |H| = N = next_pow2(len a), quotient values a/b, inverse transform and
//    unscaling.  The result q' is the polynomial of degree < N that agrees
//    with a/b on sH.  If q' has no coefficient at or above len a - len b + 1
//    then q' b - a has degree < N and N roots, so b divides a and q' is the
//    quotient; otherwise b does not divide a (error).  A coset that meets a
//    root of b is skipped for the next shift g^k (g = 5; at most deg b
//    cosets can meet a root);
//  * vanishing polynomial A = prod (X - x_i): its values at the N-th roots
//    of unity (N = next_pow2(n)) as products over the points, then one
//    inverse NTT (that gives A mod X^N - 1: for n = N the leading 1 wraps
//    into the constant term and is moved back);
//  * A'(x_i) = prod_{j != i} (x_i - x_j) directly; 1/A'(x_i) by Fermat.  A
//    zero A'(x_i) means a repeated point;
//  * interpolation f = sum_i c_i A/(X - x_i), c_i = v_i/A'(x_i): synthetic
//    division gives A/(X - x_i) = sum_k X^k sum_{m>k} A_m x_i^(m-k-1), so
//    f_k = sum_{m>k} A_m P_(m-k-1) with the power sums P_j = sum_i c_i x_i^j
//    (j < n, one product per (i, j)); the Toeplitz sum is coefficients
//    n .. 2n-1 of the product A * reverse(P), one NTT product of size
//    next_pow2(2n) against the tree's transformed A;
//  * Cauchy sums sum_{j != i} w_j/(x_i - x_j): the running pair
//    (num, den) <- (num d + w_j den, den d), d = x_i - x_j, over j != i (no
//    inversion); den ends as A'(x_i), so the sum is num / A'(x_i).  Rows
//    of weights share the den chain (1 + 2R products per pair for R rows);
//  * multipoint evaluation: Horner over chunks of coefficients, combined
//    with x^B per chunk.
//
// The pair sums, power sums and Horner chunks are quadratic in the point
// count but run as one launch over every SM, where the
// reference's remainder tree is a chain of small dependent products; for
// the supports of sparse updates (up to a few thousand points) the flat
// form is the faster one on this GPU.  Trees are capped at 2^20 points.
//
// Representation: points and denominators in Montgomery form, numerators,
// coefficients and values canonical; mont_mul(canonical, Montgomery) is the
// canonical product, so mixed products need no conversion.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "abi_util.hpp"
#include "backend.hpp"

namespace dv {

struct PolyTree {
    uint32_t n = 0, big_n = 0;  // points, max(2, next_pow2(n))
    uint32_t conv_n = 0;        // max(2, next_pow2(2 n)): the interpolation product size
    DevBuf xs;                  // Montgomery points
    DevBuf deriv, invd;         // Montgomery A'(x_i), 1/A'(x_i)
    DevBuf vanishing;           // canonical A, n + 1 coefficients
    DevBuf vanishing_hat;       // forward NTT of A padded to conv_n
};

struct PolyState {
    std::map<uint64_t, std::unique_ptr<PolyTree>> trees;
    DevBuf a, b, c, part_num, part_den, flag, shift;
    uint32_t shift_k = 0;       // the coset shift g^k held in `shift`
    NttBatch batch, batch2;
};

namespace {

constexpr int PT = 128;            // threads per block
constexpr uint32_t STAGE = 256;    // sources staged in shared memory per round
constexpr int DIV_RUN = 32;        // quotient values per thread (one inversion each)
constexpr int SCALE_RUN = 16;      // coefficients per thread in the coset scaling
constexpr uint32_t TREE_MAX = 1u << 20;
constexpr uint64_t POLY_MAX = 1ull << 24;
constexpr uint64_t ROWS_MAX = 1ull << 26;  // elements in one batched tree call

DV_INL Fr raw_one() {
    Fr r = Fr::zero();
    r.v[0] = 1;
    return r;
}

DV_INL Fr pow_u32(const Fr& base, uint32_t e) {  // Montgomery base and result
    Fr r = Fr::one();
    for (int i = 31; i >= 0; --i) {
        r = Fr::sqr(r);
        if ((e >> i) & 1) r = Fr::mul(r, base);
    }
    return r;
}

__global__ void k_to_mont(const Fr* __restrict__ in, uint64_t n, Fr* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = Fr::mul(in[i], Fr::r2());
}

__global__ void k_from_mont(const Fr* __restrict__ in, uint64_t n, Fr* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = Fr::mul(in[i], raw_one());
}

// w^k for k < big_n from the forward twiddle table (w^k, k < big_n / 2).
__global__ void k_domain(const Fr* __restrict__ tw, uint32_t big_n, Fr* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= big_n) return;
    const uint32_t half = big_n >> 1;
    out[k] = k < half ? tw[k] : Fr::neg(tw[k - half]);
}

// Partial pair sums of target t over the sources of chunk blockIdx.y:
//   den = prod (T - x_j),  num_r = sum c_(r,j) prod_(l != j) (T - x_l)
// for the R weight rows of group blockIdx.z (R = 0: den alone); SELF: the
// targets are the sources and j = t is left out.  num is canonical (the
// weights are), den Montgomery.
template <bool SELF, int R>
__global__ void __launch_bounds__(PT) k_fracsum(const Fr* __restrict__ targets, uint32_t nt,
                                                const Fr* __restrict__ xs, uint32_t n,
                                                const Fr* __restrict__ cs, uint32_t rows, uint32_t chunk,
                                                Fr* __restrict__ num_part, Fr* __restrict__ den_part) {
    constexpr int RS = R > 0 ? R : 1;
    __shared__ Fr sx[STAGE];
    __shared__ Fr sc[RS][R > 0 ? STAGE : 1];
    const uint32_t t = blockIdx.x * PT + threadIdx.x;
    const uint32_t row0 = blockIdx.z * RS;
    const uint32_t j0 = blockIdx.y * chunk, j1 = min(n, j0 + chunk);
    const bool live = t < nt;
    const Fr tv = live ? targets[t] : Fr::zero();
    Fr num[RS];
#pragma unroll
    for (int r = 0; r < RS; ++r) num[r] = Fr::zero();
    Fr den = Fr::one();
    for (uint32_t base = j0; base < j1; base += STAGE) {
        const uint32_t m = min(STAGE, j1 - base);
        __syncthreads();
        for (uint32_t s = threadIdx.x; s < m; s += PT) {
            sx[s] = xs[base + s];
#pragma unroll
            for (int r = 0; r < R; ++r)
                sc[r][s] = row0 + r < rows ? cs[(uint64_t)(row0 + r) * n + base + s] : Fr::zero();
        }
        __syncthreads();
        if (!live) continue;
        for (uint32_t s = 0; s < m; ++s) {
            if (SELF && base + s == t) continue;
            const Fr d = Fr::sub(tv, sx[s]);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const Fr::Pair p = Fr::mul2(num[r], d, sc[r][s], den);
                num[r] = Fr::add(p.r0, p.r1);
            }
            den = Fr::mul(den, d);
        }
    }
    if (!live) return;
    const uint32_t chunks = gridDim.y;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (row0 + r < rows) num_part[((uint64_t)(row0 + r) * chunks + blockIdx.y) * nt + t] = num[r];
    den_part[((uint64_t)blockIdx.z * chunks + blockIdx.y) * nt + t] = den;
}

enum FracOut { OUT_DEN_CANON, OUT_DEN_MONT, OUT_NUM_TIMES_INVD };

// Folds the chunk pairs of every (row, target): (n1, d1) + (n2, d2) =
// (n1 d2 + n2 d1, d1 d2); rows of group z = row / R share its den partials.
template <int R, int OUT>
__global__ void __launch_bounds__(PT) k_frac_combine(const Fr* __restrict__ num_part,
                                                     const Fr* __restrict__ den_part, uint32_t nt,
                                                     uint32_t chunks, uint32_t rows, const Fr* __restrict__ invd,
                                                     Fr* __restrict__ out, uint32_t* __restrict__ zero_at) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)(R > 0 ? rows : 1) * nt) return;
    const uint32_t row = (uint32_t)(i / nt), t = (uint32_t)(i % nt);
    const uint64_t dfirst = (uint64_t)(R > 0 ? row / R : 0) * chunks * nt + t;
    const uint64_t nfirst = (uint64_t)row * chunks * nt + t;
    Fr num = R > 0 ? num_part[nfirst] : Fr::zero();
    Fr den = den_part[dfirst];
    for (uint32_t c = 1; c < chunks; ++c) {
        const Fr d2 = den_part[dfirst + (uint64_t)c * nt];
        if (R > 0) {
            const Fr::Pair p = Fr::mul2(num, d2, num_part[nfirst + (uint64_t)c * nt], den);
            num = Fr::add(p.r0, p.r1);
        }
        den = Fr::mul(den, d2);
    }
    if (OUT == OUT_DEN_CANON) out[i] = Fr::mul(den, raw_one());
    if (OUT == OUT_DEN_MONT) {
        out[i] = den;
        if (den.is_zero()) atomicMin(zero_at, t);
    }
    if (OUT == OUT_NUM_TIMES_INVD) out[i] = Fr::mul(num, invd[t]);
}

constexpr int PS_G = 8;  // powers per round: one PS_G x PT tile in shared memory

// Partial power sums P_j = sum_i c_i x_i^j, c_i = v_i / A'(x_i), over the PT
// points of block blockIdx.x, for j in [blockIdx.y jt, +jt) of row
// blockIdx.z.  Each round a thread writes c_i x_i^j for PS_G consecutive j;
// then each tile row is summed by 16 threads (8 values each, columns 16
// apart so a half-warp reads consecutive elements) and a half-warp butterfly.
__global__ void __launch_bounds__(PT) k_powsum(const Fr* __restrict__ xs, uint32_t n, const Fr* __restrict__ vals,
                                               const Fr* __restrict__ invd, uint32_t jt, Fr* __restrict__ part) {
    __shared__ Fr tile[PS_G][PT];
    const uint32_t i = blockIdx.x * PT + threadIdx.x;
    const uint32_t row = blockIdx.z;
    const uint32_t j0 = blockIdx.y * jt, j1 = min(n, j0 + jt);
    Fr x = Fr::zero(), y = Fr::zero();
    if (i < n) {
        x = xs[i];
        const Fr c = Fr::mul(vals[(uint64_t)row * n + i], invd[i]);  // canonical
        y = Fr::mul(c, pow_u32(x, j0));
    }
    const uint32_t g = threadIdx.x >> 4, seg = threadIdx.x & 15;
    for (uint32_t j = j0; j < j1; j += PS_G) {
#pragma unroll
        for (int k = 0; k < PS_G; ++k) {
            tile[k][threadIdx.x] = y;
            y = Fr::mul(y, x);
        }
        __syncthreads();
        Fr acc = tile[g][seg];
#pragma unroll
        for (int k = 1; k < PT / 16; ++k) acc = Fr::add(acc, tile[g][seg + 16 * k]);
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) {
            Fr o;
#pragma unroll
            for (int w = 0; w < 8; ++w) o.v[w] = __shfl_xor_sync(0xffffffffu, acc.v[w], off);
            acc = Fr::add(acc, o);
        }
        if (seg == 0 && j + g < j1) part[((uint64_t)row * gridDim.x + blockIdx.x) * n + j + g] = acc;
        __syncthreads();
    }
}

// P_j of every row (sum of the block partials), stored reversed at
// conv[row conv_n + n - 1 - j] (the rest of the row is zero).
__global__ void __launch_bounds__(PT) k_powsum_combine(const Fr* __restrict__ part, uint32_t blocks, uint32_t n,
                                                       uint32_t rows, uint32_t conv_n, Fr* __restrict__ conv) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)rows * n) return;
    const uint32_t row = (uint32_t)(i / n), j = (uint32_t)(i % n);
    const uint64_t first = (uint64_t)row * blocks * n + j;
    Fr acc = part[first];
    for (uint32_t b = 1; b < blocks; ++b) acc = Fr::add(acc, part[first + (uint64_t)b * n]);
    conv[(uint64_t)row * conv_n + (n - 1 - j)] = acc;
}

// a[row conv_n + i] <- a[row conv_n + i] h[i] (canonical).
__global__ void k_pointwise_rows(Fr* __restrict__ a, const Fr* __restrict__ h, uint32_t conv_n, uint32_t rows) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (uint64_t)rows * conv_n) a[i] = Fr::mul(Fr::mul(a[i], Fr::r2()), h[i % conv_n]);
}

__global__ void k_invert(const Fr* __restrict__ in, uint32_t n, Fr* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = Fr::inv(in[i]);
}

// A mod (X^N - 1) -> A: for n = N the leading 1 wrapped into the constant.
__global__ void k_vanishing_fix(Fr* __restrict__ coef, uint32_t n, uint32_t big_n) {
    if (threadIdx.x || blockIdx.x) return;
    if (n == big_n) coef[0] = Fr::sub(coef[0], raw_one());
    coef[n] = raw_one();
}

// Horner of the coefficients of chunk blockIdx.y at point i (canonical
// accumulator, Montgomery point).
__global__ void __launch_bounds__(PT) k_horner(const Fr* __restrict__ xs, uint32_t n, const Fr* __restrict__ poly,
                                               uint32_t len, uint32_t chunk, Fr* __restrict__ part) {
    __shared__ Fr sp[STAGE];
    const uint32_t i = blockIdx.x * PT + threadIdx.x;
    const uint32_t row = blockIdx.z;
    const uint32_t m0 = blockIdx.y * chunk, m1 = min(len, m0 + chunk);
    const bool live = i < n;
    const Fr x = live ? xs[i] : Fr::zero();
    Fr acc = Fr::zero();
    for (uint32_t top = m1; top > m0;) {
        const uint32_t m = min(STAGE, top - m0), lo = top - m;
        __syncthreads();
        for (uint32_t s = threadIdx.x; s < m; s += PT) sp[s] = poly[(uint64_t)row * len + lo + s];
        __syncthreads();
        if (live)
            for (int s = (int)m - 1; s >= 0; --s) acc = Fr::add(Fr::mul(acc, x), sp[s]);
        top = lo;
    }
    if (live) part[((uint64_t)row * gridDim.y + blockIdx.y) * n + i] = acc;
}

__global__ void __launch_bounds__(PT) k_horner_combine(const Fr* __restrict__ part, const Fr* __restrict__ xs,
                                                       uint32_t n, uint32_t chunks, uint32_t chunk, uint32_t rows,
                                                       Fr* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)rows * n) return;
    const uint32_t row = (uint32_t)(i / n), t = (uint32_t)(i % n);
    const uint64_t first = (uint64_t)row * chunks * n + t;
    Fr r = part[first + (uint64_t)(chunks - 1) * n];
    if (chunks > 1) {
        const Fr xb = pow_u32(xs[t], chunk);
        for (int c = (int)chunks - 2; c >= 0; --c) r = Fr::add(Fr::mul(r, xb), part[first + (uint64_t)c * n]);
    }
    out[i] = r;
}

// a[i] <- a[i] b[i] (canonical in and out).
__global__ void k_pointwise(Fr* __restrict__ a, const Fr* __restrict__ b, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = Fr::mul(Fr::mul(a[i], Fr::r2()), b[i]);
}

// shift[0] = g^k, shift[1] = g^-k (Montgomery), g = 5.
__global__ void k_shift(uint32_t k, Fr* __restrict__ shift) {
    if (threadIdx.x || blockIdx.x) return;
    Fr five = Fr::zero();
    five.v[0] = 5;
    const Fr s = pow_u32(Fr::mul(five, Fr::r2()), k);
    shift[0] = s;
    shift[1] = Fr::inv(s);
}

// out[j] = in[j] s^j for j < big_n (in is zero beyond len); with `nonzero`,
// flags any nonzero output at j >= check_from.
__global__ void __launch_bounds__(PT) k_scale_powers(const Fr* __restrict__ in, uint64_t len, Fr* __restrict__ out,
                                                     uint64_t big_n, const Fr* __restrict__ s_ptr,
                                                     uint64_t check_from, uint32_t* __restrict__ nonzero) {
    const uint64_t j0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * SCALE_RUN;
    if (j0 >= big_n) return;
    const Fr s = *s_ptr;
    Fr p = pow_u32(s, (uint32_t)j0);
    bool bad = false;
    for (int r = 0; r < SCALE_RUN && j0 + r < big_n; ++r) {
        const uint64_t j = j0 + r;
        const Fr o = j < len ? Fr::mul(in[j], p) : Fr::zero();
        out[j] = o;
        if (j >= check_from && !o.is_zero()) bad = true;
        p = Fr::mul(p, s);
    }
    if (nonzero && bad) atomicOr(nonzero, 1u);
}

// a[j] <- a[j] / b[j] (canonical), one inversion per DIV_RUN values
// (Montgomery's simultaneous inversion).  Flags a zero b[j].
__global__ void __launch_bounds__(PT) k_div_values(Fr* __restrict__ a, const Fr* __restrict__ b, uint64_t big_n,
                                                   uint32_t* __restrict__ zero) {
    const uint64_t j0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * DIV_RUN;
    if (j0 >= big_n) return;
    const int m = big_n - j0 < (uint64_t)DIV_RUN ? (int)(big_n - j0) : DIV_RUN;
    Fr pre[DIV_RUN];
    Fr acc = Fr::one();
    for (int r = 0; r < m; ++r) {
        const Fr bm = Fr::mul(b[j0 + r], Fr::r2());
        if (bm.is_zero()) {
            atomicOr(zero, 1u);
            return;
        }
        pre[r] = acc;
        acc = Fr::mul(acc, bm);
    }
    Fr inv = Fr::inv(acc);
    for (int r = m - 1; r >= 0; --r) {
        const Fr bm = Fr::mul(b[j0 + r], Fr::r2());
        const Fr ib = Fr::mul(inv, pre[r]);
        inv = Fr::mul(inv, bm);
        a[j0 + r] = Fr::mul(a[j0 + r], ib);
    }
}

// ------------------------------------------------------------------ host side
PolyState& poly_state(Backend& b) {
    if (!b.poly) b.poly = std::make_shared<PolyState>();
    return *b.poly;
}

int log2_ceil(uint64_t n) {
    int k = 0;
    while ((1ull << k) < n) ++k;
    return k;
}

uint32_t blocks_for(uint64_t threads) { return (uint32_t)((threads + PT - 1) / PT); }

bool canonical_fr(const uint8_t* p) {
    static const uint64_t R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                                  0x30644e72e131a029ull};
    uint64_t v[4];
    memcpy(v, p, 32);
    for (int i = 3; i >= 0; --i) {
        if (v[i] < R[i]) return true;
        if (v[i] > R[i]) return false;
    }
    return false;
}

void require_canonical(const uint8_t* p, uint64_t count, const char* what) {
    for (uint64_t i = 0; i < count; ++i)
        if (!canonical_fr(p + 32 * i))
            throw InvalidArgument(std::string("non-canonical ") + what + " at index " + std::to_string(i));
}

bool zero_fr(const uint8_t* p) {
    for (int i = 0; i < 32; ++i)
        if (p[i]) return false;
    return true;
}

// Length after the reference's trim (domain.rs:339-346): at least 1.
uint64_t trimmed(const uint8_t* p, uint64_t len) {
    while (len > 1 && zero_fr(p + 32 * (len - 1))) --len;
    return len ? len : 1;
}

// Source chunks for `targets` x `rows` threads over n sources: enough
// threads for every SM, at least 32 sources per chunk.
uint32_t source_chunk(uint64_t targets, uint32_t rows, uint32_t n) {
    const uint64_t goal = (uint64_t)sm_count() * 1024;
    const uint64_t threads = (uint64_t)blocks_for(targets) * PT * rows;
    uint64_t chunks = (goal + threads - 1) / threads;
    chunks = std::min<uint64_t>(chunks, std::max<uint64_t>(1, n / 32));
    chunks = std::max<uint64_t>(1, std::min<uint64_t>(chunks, 65535));
    const uint64_t chunk = (n + chunks - 1) / chunks;
    return (uint32_t)std::max<uint64_t>(1, chunk);
}

// Pair sums over all sources for every (row, target), folded into `out`;
// R weight rows per thread group (R = 0: den alone).
template <bool SELF, int R, int OUT>
void fracsum(PolyState& ps, const Fr* targets, uint32_t nt, const Fr* xs, uint32_t n, const Fr* cs, uint32_t rows,
             const Fr* invd, Fr* out, uint32_t* zero_at, cudaStream_t st) {
    const uint32_t groups = R > 0 ? (rows + R - 1) / R : 1;
    const uint32_t chunk = source_chunk(nt, groups, n);
    const uint32_t chunks = n ? (n + chunk - 1) / chunk : 1;
    Fr* pn = R > 0 ? ps.part_num.as<Fr>((uint64_t)rows * chunks * nt) : nullptr;
    Fr* pd = ps.part_den.as<Fr>((uint64_t)groups * chunks * nt);
    k_fracsum<SELF, R><<<dim3(blocks_for(nt), chunks, groups), PT, 0, st>>>(targets, nt, xs, n, cs, rows, chunk, pn,
                                                                           pd);
    DV_LAUNCH();
    k_frac_combine<R, OUT><<<blocks_for((uint64_t)(R > 0 ? rows : 1) * nt), PT, 0, st>>>(pn, pd, nt, chunks, rows,
                                                                                         invd, out, zero_at);
    DV_LAUNCH();
}

// Transforms `rows` consecutive vectors of 2^logn canonical elements in place
// (one persistent batch launch; ntt_batch_check after the stream is done).
void ntt_rows(Backend& b, NttBatch& batch, Fr* data, int logn, uint32_t rows, int kind, cudaStream_t st) {
    std::vector<NttBatchItem> items(rows);
    for (uint32_t r = 0; r < rows; ++r) {
        uint8_t* p = reinterpret_cast<uint8_t*>(data + ((uint64_t)r << logn));
        items[r] = NttBatchItem{p, p, logn, kind};
    }
    ntt_batch_prepare(b.ntt, batch, items, st);
    ntt_batch_enqueue(batch, st);
}

PolyTree& tree_of(PolyState& ps, uint64_t h) {
    auto it = ps.trees.find(h);
    if (it == ps.trees.end()) throw InvalidArgument("unknown subproduct tree handle");
    return *it->second;
}

// SubproductTree::new (fast.rs:38-62): vanishing polynomial (and its
// transform of size conv_n) and inverse derivative values of `count`
// distinct canonical points.
std::unique_ptr<PolyTree> tree_build(Backend& b, PolyState& ps, const uint8_t* points, uint32_t count,
                                     cudaStream_t st) {
    auto t = std::make_unique<PolyTree>();
    t->n = count;
    t->big_n = (uint32_t)std::max<uint64_t>(2, 1ull << log2_ceil(count));
    t->conv_n = (uint32_t)std::max<uint64_t>(2, 1ull << log2_ceil(2ull * count));
    const int logn = log2_ceil(t->big_n);
    Fr* van = t->vanishing.as<Fr>((uint64_t)t->big_n + 1);
    if (count == 0) {
        const uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0};
        DV_CUDA(cudaMemcpyAsync(van, one, 32, cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaStreamSynchronize(st));
        return t;
    }
    Fr* stage = ps.a.as<Fr>(std::max<uint64_t>(count, t->big_n));
    DV_CUDA(cudaMemcpyAsync(stage, points, 32ull * count, cudaMemcpyHostToDevice, st));
    Fr* xs = t->xs.as<Fr>(count);
    k_to_mont<<<blocks_for(count), PT, 0, st>>>(stage, count, xs);
    DV_LAUNCH();
    Fr* dom = stage;  // the points are converted: reuse the staging buffer for w^k
    const Fr* tw = ntt_tables(b.ntt, logn, NTT_FORWARD, st).tw.as<Fr>(1);
    k_domain<<<blocks_for(t->big_n), PT, 0, st>>>(tw, t->big_n, dom);
    DV_LAUNCH();
    fracsum<false, 0, OUT_DEN_CANON>(ps, dom, t->big_n, xs, count, nullptr, 1, nullptr, van, nullptr, st);
    ntt_rows(b, ps.batch, van, logn, 1, NTT_INVERSE, st);
    k_vanishing_fix<<<1, 32, 0, st>>>(van, count, t->big_n);
    DV_LAUNCH();
    Fr* hat = t->vanishing_hat.as<Fr>(t->conv_n);
    DV_CUDA(cudaMemsetAsync(hat, 0, 32ull * t->conv_n, st));
    DV_CUDA(cudaMemcpyAsync(hat, van, 32ull * (count + 1), cudaMemcpyDeviceToDevice, st));
    ntt_rows(b, ps.batch2, hat, log2_ceil(t->conv_n), 1, NTT_FORWARD, st);
    uint32_t* zero_at = ps.flag.as<uint32_t>(1);
    DV_CUDA(cudaMemsetAsync(zero_at, 0xff, sizeof(uint32_t), st));
    Fr* deriv = t->deriv.as<Fr>(count);
    fracsum<true, 0, OUT_DEN_MONT>(ps, xs, count, xs, count, nullptr, 1, nullptr, deriv, zero_at, st);
    k_invert<<<blocks_for(count), PT, 0, st>>>(deriv, count, t->invd.as<Fr>(count));
    DV_LAUNCH();
    ntt_batch_check(ps.batch, st);
    ntt_batch_check(ps.batch2, st);
    if (read_err_word(b, zero_at, st) != 0xffffffffu) throw InvalidArgument("duplicate interpolation point");
    return t;
}

// Cauchy sums of `rows` weight rows (device, canonical) into out (rows x n).
void cauchy_rows(PolyState& ps, PolyTree& t, const Fr* w, uint32_t rows, Fr* out, cudaStream_t st) {
    const Fr* xs = t.xs.view<Fr>();
    const Fr* invd = t.invd.view<Fr>();
    if (rows >= 4)
        fracsum<true, 4, OUT_NUM_TIMES_INVD>(ps, xs, t.n, xs, t.n, w, rows, invd, out, nullptr, st);
    else if (rows == 3)
        fracsum<true, 3, OUT_NUM_TIMES_INVD>(ps, xs, t.n, xs, t.n, w, rows, invd, out, nullptr, st);
    else if (rows == 2)
        fracsum<true, 2, OUT_NUM_TIMES_INVD>(ps, xs, t.n, xs, t.n, w, rows, invd, out, nullptr, st);
    else
        fracsum<true, 1, OUT_NUM_TIMES_INVD>(ps, xs, t.n, xs, t.n, w, rows, invd, out, nullptr, st);
}

// Interpolation of `rows` value rows (device, canonical): the coefficients
// of row r end up at conv[r conv_n + n ..], n of them.
Fr* interpolate_rows(Backend& b, PolyState& ps, PolyTree& t, const Fr* vals, uint32_t rows, cudaStream_t st) {
    const uint32_t n = t.n;
    const uint32_t blocks = blocks_for(n);
    // j tiles: enough blocks for every SM, at least 128 powers per tile (the
    // tile's starting power x^j0 costs about 2 log2 j0 products)
    const uint64_t goal = (uint64_t)sm_count() * 8;
    uint64_t tiles = (goal + (uint64_t)blocks * rows - 1) / ((uint64_t)blocks * rows);
    tiles = std::max<uint64_t>(1, std::min<uint64_t>(tiles, (n + 127) / 128));
    uint32_t jt = (uint32_t)((n + tiles - 1) / tiles);
    jt = (jt + PS_G - 1) / PS_G * PS_G;
    tiles = (n + jt - 1) / jt;
    Fr* part = ps.part_num.as<Fr>((uint64_t)rows * blocks * n);
    k_powsum<<<dim3(blocks, (uint32_t)tiles, rows), PT, 0, st>>>(t.xs.view<Fr>(), n, vals, t.invd.view<Fr>(), jt,
                                                                 part);
    DV_LAUNCH();
    Fr* conv = ps.c.as<Fr>((uint64_t)rows * t.conv_n);
    DV_CUDA(cudaMemsetAsync(conv, 0, 32ull * rows * t.conv_n, st));
    k_powsum_combine<<<blocks_for((uint64_t)rows * n), PT, 0, st>>>(part, blocks, n, rows, t.conv_n, conv);
    DV_LAUNCH();
    const int logc = log2_ceil(t.conv_n);
    ntt_rows(b, ps.batch, conv, logc, rows, NTT_FORWARD, st);
    k_pointwise_rows<<<blocks_for((uint64_t)rows * t.conv_n), PT, 0, st>>>(conv, t.vanishing_hat.view<Fr>(),
                                                                           t.conv_n, rows);
    DV_LAUNCH();
    ntt_rows(b, ps.batch2, conv, logc, rows, NTT_INVERSE, st);
    return conv;
}

void copy_out(void* dst, const void* src, uint64_t bytes, cudaStream_t st) {
    if (bytes) DV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
}

}  // namespace
}  // namespace dv

using namespace dv;

// ============================================================ products
extern "C" int dvgpu_bn254_poly_multiply(void* opaque, const uint8_t* left, size_t left_len, const uint8_t* right,
                                         size_t right_len, uint8_t* result, size_t result_cap, size_t* result_len,
                                         char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(result && result_len && (left || !left_len) && (right || !right_len), "invalid product buffers");
        const uint64_t out_len = (left_len && right_len) ? (uint64_t)left_len + right_len - 1 : 1;
        require(result_cap >= out_len, "product result buffer too small");
        require(out_len <= POLY_MAX, "polynomial product longer than 2^24 coefficients");
        require_canonical(left, left_len, "left coefficient");
        require_canonical(right, right_len, "right coefficient");
        if (!left_len || !right_len) {  // fast.rs:214: an empty operand gives the zero polynomial
            memset(result, 0, 32);
            *result_len = 1;
            return;
        }
        PolyState& ps = poly_state(b);
        const cudaStream_t st = b.stream;
        const int logn = std::max(1, log2_ceil(out_len));
        const uint64_t big_n = 1ull << logn;
        Fr* two = ps.a.as<Fr>(2 * big_n);
        Fr* l = two;
        Fr* r = two + big_n;
        DV_CUDA(cudaMemsetAsync(two, 0, 64 * big_n, st));
        DV_CUDA(cudaMemcpyAsync(l, left, 32 * left_len, cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaMemcpyAsync(r, right, 32 * right_len, cudaMemcpyHostToDevice, st));
        ntt_rows(b, ps.batch, two, logn, 2, NTT_FORWARD, st);
        k_pointwise<<<blocks_for(big_n), PT, 0, st>>>(l, r, big_n);
        DV_LAUNCH();
        ntt_batch_check(ps.batch, st);
        ntt_rows(b, ps.batch, l, logn, 1, NTT_INVERSE, st);
        copy_out(result, l, 32 * out_len, st);
        ntt_batch_check(ps.batch, st);  // synchronises
        *result_len = trimmed(result, out_len);
    });
}

// ============================================================ exact division
extern "C" int dvgpu_bn254_poly_divide_exact(void* opaque, const uint8_t* numerator, size_t numerator_len,
                                             const uint8_t* denominator, size_t denominator_len, uint8_t* quotient,
                                             size_t quotient_cap, size_t* quotient_len, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(quotient && quotient_len && (numerator || !numerator_len) && (denominator || !denominator_len),
                "invalid division buffers");
        require(quotient_cap >= std::max<size_t>(1, numerator_len), "quotient buffer too small");
        require(numerator_len <= POLY_MAX && denominator_len <= POLY_MAX,
                "polynomial division operands longer than 2^24 coefficients");
        require_canonical(numerator, numerator_len, "numerator coefficient");
        require_canonical(denominator, denominator_len, "denominator coefficient");
        // div_rem_impl (fast.rs:163-170): trim both, reject a zero divisor.
        const uint64_t nl = numerator_len ? trimmed(numerator, numerator_len) : 1;
        const uint64_t dl = denominator_len ? trimmed(denominator, denominator_len) : 1;
        const bool num_zero = !numerator_len || (nl == 1 && zero_fr(numerator));
        require(denominator_len && !(dl == 1 && zero_fr(denominator)), "cannot divide by zero polynomial");
        if (nl < dl || num_zero) {  // quotient 0, remainder = numerator
            require(num_zero, "polynomial division has a nonzero remainder");
            memset(quotient, 0, 32);
            *quotient_len = 1;
            return;
        }
        const uint64_t qlen = nl - dl + 1;
        PolyState& ps = poly_state(b);
        const cudaStream_t st = b.stream;
        const int logn = std::max(1, log2_ceil(nl));
        const uint64_t big_n = 1ull << logn;
        Fr* orig = ps.b.as<Fr>(2 * big_n);  // numerator | denominator coefficients
        Fr* work = ps.a.as<Fr>(2 * big_n);  // their coset values
        Fr* shift = ps.shift.as<Fr>(2);  // grow-only: allocated once, so a cached shift stays valid
        uint32_t* flag = ps.flag.as<uint32_t>(1);
        DV_CUDA(cudaMemcpyAsync(orig, numerator, 32 * nl, cudaMemcpyHostToDevice, st));
        DV_CUDA(cudaMemcpyAsync(orig + big_n, denominator, 32 * dl, cudaMemcpyHostToDevice, st));
        const uint32_t scale_blocks = blocks_for((big_n + SCALE_RUN - 1) / SCALE_RUN);
        // A coset meets at most dl - 1 roots of the divisor, so dl shifts suffice.
        for (uint32_t k = 1;; ++k) {
            require(k <= dl, "no coset avoids the divisor's roots");
            if (ps.shift_k != k) {
                k_shift<<<1, 32, 0, st>>>(k, shift);
                DV_LAUNCH();
                ps.shift_k = k;
            }
            k_scale_powers<<<scale_blocks, PT, 0, st>>>(orig, nl, work, big_n, shift, big_n, nullptr);
            DV_LAUNCH();
            k_scale_powers<<<scale_blocks, PT, 0, st>>>(orig + big_n, dl, work + big_n, big_n, shift, big_n, nullptr);
            DV_LAUNCH();
            ntt_rows(b, ps.batch, work, logn, 2, NTT_FORWARD, st);
            DV_CUDA(cudaMemsetAsync(flag, 0, sizeof(uint32_t), st));
            k_div_values<<<blocks_for((big_n + DIV_RUN - 1) / DIV_RUN), PT, 0, st>>>(work, work + big_n, big_n, flag);
            DV_LAUNCH();
            ntt_batch_check(ps.batch, st);
            if (read_err_word(b, flag, st) == 0) break;
        }
        ntt_rows(b, ps.batch, work, logn, 1, NTT_INVERSE, st);
        DV_CUDA(cudaMemsetAsync(flag, 0, sizeof(uint32_t), st));
        // unscale by s^-j into the spare half and flag any coefficient at or above qlen
        k_scale_powers<<<scale_blocks, PT, 0, st>>>(work, big_n, work + big_n, big_n, shift + 1, qlen, flag);
        DV_LAUNCH();
        copy_out(quotient, work + big_n, 32 * qlen, st);
        ntt_batch_check(ps.batch, st);
        if (read_err_word(b, flag, st) != 0) throw InvalidArgument("polynomial division has a nonzero remainder");
        *quotient_len = trimmed(quotient, qlen);
    });
}

// ============================================================ subproduct trees
extern "C" int dvgpu_bn254_tree_create(void* opaque, const uint8_t* points, size_t count, uint64_t* tree,
                                       char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(tree && (points || !count), "invalid subproduct tree arguments");
        require(count <= TREE_MAX, "subproduct tree holds at most 2^20 points");
        require_canonical(points, count, "interpolation point");
        PolyState& ps = poly_state(b);
        auto t = tree_build(b, ps, points, (uint32_t)count, b.stream);
        const uint64_t h = b.next_handle++;
        ps.trees[h] = std::move(t);
        *tree = h;
    });
}

extern "C" int dvgpu_bn254_tree_destroy(void* opaque, uint64_t tree, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PolyState& ps = poly_state(b);
        tree_of(ps, tree);
        DV_CUDA(cudaStreamSynchronize(b.stream));
        ps.trees.erase(tree);
    });
}

extern "C" int dvgpu_bn254_tree_vanishing(void* opaque, uint64_t tree, uint8_t* coefficients, size_t capacity,
                                          size_t* length, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PolyTree& t = tree_of(poly_state(b), tree);
        require(coefficients && length && capacity >= (size_t)t.n + 1, "vanishing polynomial buffer too small");
        copy_out(coefficients, t.vanishing.view<Fr>(), 32ull * (t.n + 1), b.stream);
        DV_CUDA(cudaStreamSynchronize(b.stream));
        *length = t.n + 1;
    });
}

extern "C" int dvgpu_bn254_tree_inverse_derivatives(void* opaque, uint64_t tree, uint8_t* values, size_t capacity,
                                                    char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PolyState& ps = poly_state(b);
        PolyTree& t = tree_of(ps, tree);
        require((values || !t.n) && capacity >= t.n, "inverse derivative buffer too small");
        if (!t.n) return;
        Fr* out = ps.c.as<Fr>(t.n);
        k_from_mont<<<blocks_for(t.n), PT, 0, b.stream>>>(t.invd.view<Fr>(), t.n, out);
        DV_LAUNCH();
        copy_out(values, out, 32ull * t.n, b.stream);
        DV_CUDA(cudaStreamSynchronize(b.stream));
    });
}

// SubproductTree::multipoint_eval (fast.rs:73-84): `rows` polynomials of
// `length` coefficients each, values at the tree's points in point order.
extern "C" int dvgpu_bn254_tree_evaluate(void* opaque, uint64_t tree, const uint8_t* polynomials, size_t length,
                                         size_t rows, uint8_t* values, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PolyState& ps = poly_state(b);
        PolyTree& t = tree_of(ps, tree);
        require(rows >= 1 && rows <= 65535 && (polynomials || !length) && (values || !t.n),
                "invalid evaluation arguments");
        require(length <= POLY_MAX && (uint64_t)rows * std::max<uint64_t>(length, t.n) <= ROWS_MAX,
                "evaluation batch larger than 2^26 elements");
        require_canonical(polynomials, (uint64_t)length * rows, "polynomial coefficient");
        if (!t.n) return;
        const uint64_t total = (uint64_t)rows * t.n;
        if (!length) {
            memset(values, 0, 32 * total);
            return;
        }
        const cudaStream_t st = b.stream;
        Fr* poly = ps.a.as<Fr>((uint64_t)rows * length);
        DV_CUDA(cudaMemcpyAsync(poly, polynomials, 32ull * rows * length, cudaMemcpyHostToDevice, st));
        const uint32_t chunk = source_chunk(t.n, (uint32_t)rows, (uint32_t)length);
        const uint32_t chunks = (uint32_t)((length + chunk - 1) / chunk);
        Fr* part = ps.part_num.as<Fr>(total * chunks);
        k_horner<<<dim3(blocks_for(t.n), chunks, (uint32_t)rows), PT, 0, st>>>(t.xs.view<Fr>(), t.n, poly,
                                                                               (uint32_t)length, chunk, part);
        DV_LAUNCH();
        Fr* out = ps.c.as<Fr>(total);
        k_horner_combine<<<blocks_for(total), PT, 0, st>>>(part, t.xs.view<Fr>(), t.n, chunks, chunk, (uint32_t)rows,
                                                           out);
        DV_LAUNCH();
        copy_out(values, out, 32 * total, st);
        DV_CUDA(cudaStreamSynchronize(st));
    });
}

// SubproductTree::interpolate (fast.rs:90-116): `rows` value vectors of
// `count` (= points) entries; coefficients rows x max(1, count), trimmed
// lengths in `lengths`.
extern "C" int dvgpu_bn254_tree_interpolate(void* opaque, uint64_t tree, const uint8_t* values, size_t count,
                                            size_t rows, uint8_t* coefficients, size_t* lengths, char* error,
                                            size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PolyState& ps = poly_state(b);
        PolyTree& t = tree_of(ps, tree);
        require(count == t.n, "interpolation value count differs from points");
        require(rows >= 1 && rows <= 65535 && (values || !count) && coefficients && lengths,
                "invalid interpolation arguments");
        require((uint64_t)rows * t.conv_n <= ROWS_MAX, "interpolation batch larger than 2^26 elements");
        require_canonical(values, (uint64_t)count * rows, "interpolation value");
        if (!t.n) {
            memset(coefficients, 0, 32 * rows);
            for (size_t r = 0; r < rows; ++r) lengths[r] = 1;
            return;
        }
        const cudaStream_t st = b.stream;
        Fr* vals = ps.b.as<Fr>((uint64_t)rows * t.n);
        DV_CUDA(cudaMemcpyAsync(vals, values, 32ull * rows * t.n, cudaMemcpyHostToDevice, st));
        const Fr* conv = interpolate_rows(b, ps, t, vals, (uint32_t)rows, st);
        DV_CUDA(cudaMemcpy2DAsync(coefficients, 32ull * t.n, conv + t.n, 32ull * t.conv_n, 32ull * t.n, rows,
                                  cudaMemcpyDeviceToHost, st));
        ntt_batch_check(ps.batch, st);
        ntt_batch_check(ps.batch2, st);  // synchronises
        for (size_t r = 0; r < rows; ++r) lengths[r] = trimmed(coefficients + 32ull * t.n * r, t.n);
    });
}

// SubproductTree::cauchy_sums (fast.rs:118-139): sum_{j != i} w_j/(x_i - x_j)
// for `rows` weight vectors of `count` (= points) entries.
extern "C" int dvgpu_bn254_tree_cauchy_sums(void* opaque, uint64_t tree, const uint8_t* weights, size_t count,
                                            size_t rows, uint8_t* sums, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PolyState& ps = poly_state(b);
        PolyTree& t = tree_of(ps, tree);
        require(count == t.n, "Cauchy weight count differs from points");
        require(rows >= 1 && rows <= 65535 && ((weights && sums) || !count), "invalid Cauchy arguments");
        require((uint64_t)rows * t.n <= ROWS_MAX, "Cauchy batch larger than 2^26 elements");
        require_canonical(weights, (uint64_t)count * rows, "Cauchy weight");
        if (!t.n) return;
        const cudaStream_t st = b.stream;
        const uint64_t total = (uint64_t)rows * t.n;
        Fr* w = ps.b.as<Fr>(total);
        DV_CUDA(cudaMemcpyAsync(w, weights, 32 * total, cudaMemcpyHostToDevice, st));
        Fr* out = ps.c.as<Fr>(total);
        cauchy_rows(ps, t, w, (uint32_t)rows, out, st);
        copy_out(sums, out, 32 * total, st);
        DV_CUDA(cudaStreamSynchronize(st));
    });
}
