// BN254 optimal ate pairing and pairing-product checks on sm_100a.
//
// The verifier's checks (crates/protocol/src/verification.rs:37-144):
// PairingChecks::equal / equal_prepared / product_equal reduce one equation
// to prod_k e(P_k, Q_k) = 1 (right-hand G1 points negated by the caller),
// computed by Bn254::multi_miller_loop and final_exponentiation.  Here a
// launch takes many equations: a group of six lanes runs the Miller loop of
// one term (or, with prepared G2 points in large batches, the multi-Miller
// loop of one equation), then a group per equation multiplies its terms'
// values and runs the final exponentiation.  The reference's native Miller probe
// (native/include/dynaverse_bn254_miller.h) is a diagnostic of line traces
// and is not reproduced.
//
// Fq12 = Fq2[w]/(w^6 - xi), xi = 9 + u, held by six lanes: lane k owns the
// coefficient of w^k.  A product is a three-term Karatsuba over
// Fq4 = Fq2[w^3], one Fq4 product (three Fq2 products) per lane from
// shuffled operands; a square the same with Fq4 squares; the sparse line
// product is c_k = sum_i f_i l_(k-i) over the line's three coefficients,
// three Fq2 products per lane; the q-power Frobenius
// is conj(a_k) xi^(k(q-1)/6) per lane; f^(q^6) negates the odd lanes.  The
// serialised GT element uses the tower Fq12 = Fq6[w]/(w^2 - v), Fq6 =
// Fq2[v]/(v^3 - xi), v = w^2: c0 = (w^0, w^2, w^4), c1 = (w^1, w^3, w^5).
//
// Miller loop over the NAF of 6z + 2 (z the BN seed), then the lines to
// pi(Q) and -pi^2(Q).  T is kept in Jacobian coordinates on the twist
// E': y^2 = x^3 + 3/xi, untwisted by (x, y) -> (x w^2, y w^3).  The line
// through T (slope lam) at P = (xp, yp) is yp - lam xp w + (lam xT - yT) w^3;
// each step multiplies it by a nonzero Fq2 factor (killed by the final
// exponentiation, since Fq2* lies in the kernel of q^6 - 1).  The products
// of a step are spread over the group's lanes level by level:
//   doubling, x = X/Z^2, y = Y/Z^3, factor 2 Y Z^3:
//     (2 Y Z^3 yp) + (-3 X^2 Z^2 xp) w + (3 X^3 - 2 Y^2) w^3
//   addition of affine S = (xs, ys), H = xs Z^2 - X, R = ys Z^3 - Y, factor 2 Z H:
//     (2 Z H yp) + (-2 R xp) w + (2 R xs - 2 Z H ys) w^3
// with the doubling and mixed-addition formulas dbl-2009-l and
// madd-2007-bl (Explicit-Formulas Database) for the point itself.
//
// Final exponentiation: the easy part (q^6 - 1)(q^2 + 1) by conjugation,
// inversion and a q^2 Frobenius, then the exponent
// 2z(6z^2 + 3z + 1)(q^4 - q^2 + 1)/r, whose base-q digits are
//   l0 = 12z^3 + 12z^2 + 6z + 1, l1 = 12z^3 + 6z^2 + 4z,
//   l2 = 12z^3 + 6z^2 + 6z,      l3 = 12z^3 + 6z^2 + 4z - 1
// (Fuentes-Castaneda, Knapp and Rodriguez-Henriquez, "Faster hashing to
// G2", SAC 2011), from a = f^z, b = a^z, c = b^z:
//   T = c^12 b^6, f^l1 = T a^4, f^l2 = T a^6, f^l3 = f^l1 conj(f),
//   f^l0 = c^12 b^12 a^6 f, result = f^l0 (f^l1)^q (f^l2)^(q^2) (f^l3)^(q^3).
// conj is the inverse after the easy part (the result is in the
// cyclotomic subgroup, where squares take the Granger-Scott form); the easy part's inverse is conj(f) / N with N =
// f conj(f) in Fq6 inverted in every lane.  A verdict is result == 1; the
// value written for a single pairing is the GT element in the tower order
// above, canonical.
#include <cstring>
#include <map>
#include <memory>
#include <unordered_map>
#include <string>
#include <vector>

#include "abi_util.hpp"
#include "backend.hpp"
#include "engine.hpp"

namespace dv {
namespace {

struct Fq6 {
    Fq2 c0, c1, c2;
};

// xi^(j (q-1)/6), j = 0..5, Montgomery (c0, c1).
__device__ __constant__ uint32_t FROB1[6][2][8] = {
    {{0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u, 0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u},
     {0x00000000u, 0x00000000u, 0x00000000u, 0x00000000u, 0x00000000u, 0x00000000u, 0x00000000u, 0x00000000u}},
    {{0x33144907u, 0xaf9ba696u, 0x87afb78au, 0xca6b1d73u, 0xf08a2087u, 0x11bded5eu, 0x1a1f3a7cu, 0x02f34d75u},
     {0x4c492d72u, 0xa222ae23u, 0x565de15bu, 0xd00f02a4u, 0x53dfc926u, 0xdc2ff3a2u, 0xb3899551u, 0x10a75716u}},
    {{0x4563ab30u, 0xb5773b10u, 0xa9aa6454u, 0x347f91c8u, 0x242e0991u, 0x7a007127u, 0x118214ecu, 0x1956bcd8u},
     {0xa0aa4757u, 0x6e849f1eu, 0x89f89141u, 0xaa1c7b6du, 0xfae0ca3au, 0xb6e713cdu, 0x4e82ebc3u, 0x26694fbbu}},
    {{0x2936b629u, 0xe4bbdd0cu, 0xe133bacbu, 0xbb30f162u, 0xf9645366u, 0x31a9d1b6u, 0xa500f8ddu, 0x253570beu},
     {0x5ffe77c7u, 0xa1d77ce4u, 0x7826d1dbu, 0x07affd11u, 0xbb7edc6bu, 0x6d16bd27u, 0x85defeccu, 0x2c872002u}},
    {{0x843abe92u, 0x7361d77fu, 0x273411fbu, 0xa5bb2bd3u, 0x4b3e2399u, 0x9c941f31u, 0xbb9fd3ecu, 0x15df9cddu},
     {0x4bd8c949u, 0x5dddfd15u, 0xa4445b60u, 0x62cb29a5u, 0x0c7dd2b9u, 0x37bc870au, 0x3171f0fdu, 0x24830a9du}},
    {{0x41690fe7u, 0xc970692fu, 0x27694b0bu, 0xe2403421u, 0x83c459e8u, 0x32bee66bu, 0x0ab08841u, 0x12aabcedu},
     {0x40aebfa9u, 0x0d485d23u, 0xab2fcc57u, 0x05193418u, 0x8a4910f5u, 0xd3b0a40bu, 0x35d2925au, 0x2f21ebb5u}}};
// |xi^(j (q-1)/6)|^2 = xi^(j (q^2-1)/6) in Fq, Montgomery.
__device__ __constant__ uint32_t FROB2[6][8] = {
    {0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u, 0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u},
    {0x00fa1bf2u, 0xca8d8005u, 0x68b39769u, 0xf0c5d614u, 0xad0d4418u, 0x0e201271u, 0xbad856e6u, 0x04290f65u},
    {0x13e80b9cu, 0x3350c88eu, 0xdb5e56b9u, 0x7dce557cu, 0xb615564au, 0x6001b4b8u, 0x020217e0u, 0x2682e617u},
    {0x12edefaau, 0x68c34889u, 0x72aabf4fu, 0x8d087f68u, 0x09081231u, 0x51e1a247u, 0x4729c0fau, 0x2259d6b1u},
    {0xd782e155u, 0x71930c11u, 0xffbe3323u, 0xa6bb947cu, 0xd4741444u, 0xaa303344u, 0x26594943u, 0x2c3b3f0du},
    {0xc494f1abu, 0x08cfc388u, 0x8d1373d4u, 0x19b31514u, 0xcb6c0213u, 0x584e90fdu, 0xdf2f8849u, 0x09e1685bu}};
// NAF of 6z + 2, most significant digit first.
__device__ __constant__ int8_t NAF_6Z2[66] = {1, 0, -1, 0, 1, 0, 0, 0, -1, 0, -1, 0, 0, 0, -1, 0, 1, 0, -1, 0, 0, -1, 0, 0, 0, 0, 0, 1, 0, 0, -1, 0, 1, 0, 0, -1, 0, 0, 0, 0, -1, 0, 1, 0, 0, 0, -1, 0, -1, 0, 0, 1, 0, 0, 0, -1, 0, 0, -1, 0, 1, 0, 1, 0, 0, 0};
constexpr int NAF_LEN = 66;
// Width-4 NAF of z, most significant digit first: 14 odd digits in
// {+-1, +-3, +-5, +-7} (against 24 in the plain NAF and 28 binary).
__device__ __constant__ int8_t WNAF_Z[63] = {1, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, -3, 0, 0, 0, 3, 0, 0, 0, 0, 5, 0, 0, 0, -5, 0, 0, 0, -3, 0, 0, 0, 1, 0, 0, 0, 0, 5, 0, 0, 0, 0, 7, 0, 0, 0, -7, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, -1, 0, 0, 0, 1};
constexpr int WNAF_Z_LEN = 63;

DV_INL Fq load_fq(const uint32_t* w) {
    Fq r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = w[i];
    return r;
}
DV_INL Fq2 frob1(int j) { return {load_fq(FROB1[j][0]), load_fq(FROB1[j][1])}; }
DV_INL Fq frob2(int j) { return load_fq(FROB2[j]); }

DV_INL Fq mul9(const Fq& a) { return Fq::add(Fq::dbl(Fq::dbl(Fq::dbl(a))), a); }
// (a0 + a1 u)(9 + u) = (9 a0 - a1) + (a0 + 9 a1) u
DV_INL Fq2 mul_xi(const Fq2& a) { return {Fq::sub(mul9(a.c0), a.c1), Fq::add(a.c0, mul9(a.c1))}; }


// 1 / a in Fq6 (one Fq inversion).
__device__ __noinline__ Fq6 f6_inv(const Fq6& a) {
    const Fq2 t0 = Fq2::sub(Fq2::sqr(a.c0), mul_xi(Fq2::mul(a.c1, a.c2)));
    const Fq2 t1 = Fq2::sub(mul_xi(Fq2::sqr(a.c2)), Fq2::mul(a.c0, a.c1));
    const Fq2 t2 = Fq2::sub(Fq2::sqr(a.c1), Fq2::mul(a.c0, a.c2));
    const Fq2 d = Fq2::add(Fq2::mul(a.c0, t0), mul_xi(Fq2::add(Fq2::mul(a.c2, t1), Fq2::mul(a.c1, t2))));
    const Fq2 di = Fq2::inv(d);
    return {Fq2::mul(t0, di), Fq2::mul(t1, di), Fq2::mul(t2, di)};
}

// ------------------------------------------------------------------ lane groups
// One Fq12 lives in a group of GL = 6 lanes: lane k holds the Fq2
// coefficient of w^k (w^6 = xi).  A warp holds 5 groups (lanes 30, 31 run
// along on copies and write nothing); every group in a warp executes the
// same instruction stream, so the shuffles below always see full warps.
constexpr unsigned FULL = 0xffffffffu;
constexpr int GL = 6;
constexpr int GROUPS_PER_WARP = 5;

DV_INL Fq shfl_fq(const Fq& a, int src) {
    Fq r;
#pragma unroll
    for (int w = 0; w < 8; ++w) r.v[w] = __shfl_sync(FULL, a.v[w], src);
    return r;
}
DV_INL Fq2 shfl2(const Fq2& a, int src) { return {shfl_fq(a.c0, src), shfl_fq(a.c1, src)}; }
DV_INL int mod6(int x) { return x < 0 ? x + 6 : (x >= 6 ? x - 6 : x); }

// n Fq2 products (Karatsuba, 3 base products each) with their 3n base
// products issued two at a time (one out-of-line body interleaves the two
// chains, which a lone warp needs to hide the multiply latency).
template <int N>
DV_INL void fq2_mul_n(const Fq2* a, const Fq2* b, Fq2* out) {
    constexpr int M = 3 * N, G = (M + 1) / 2;
    Fq x[2 * G], y[2 * G], z[2 * G];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        x[3 * i] = a[i].c0; y[3 * i] = b[i].c0;
        x[3 * i + 1] = a[i].c1; y[3 * i + 1] = b[i].c1;
        x[3 * i + 2] = Fq::add(a[i].c0, a[i].c1); y[3 * i + 2] = Fq::add(b[i].c0, b[i].c1);
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (2 * g + 1 < M) {
            const Fq::Pair q = Fq::mul2(x[2 * g], y[2 * g], x[2 * g + 1], y[2 * g + 1]);
            z[2 * g] = q.r0;
            z[2 * g + 1] = q.r1;
        } else {
            z[2 * g] = Fq::mul(x[2 * g], y[2 * g]);
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
        out[i] = {Fq::sub(z[3 * i], z[3 * i + 1]), Fq::sub(Fq::sub(z[3 * i + 2], z[3 * i]), z[3 * i + 1])};
}

// Products and squares by Karatsuba over Fq4 = Fq2[t]/(t^2 - xi), t = w^3:
// f = F0 + F1 w + F2 w^2 with F_i = f_i + f_(i+3) t and w^3 = t.  The six
// Fq4 products of a three-term Karatsuba, one per lane (three Fq2 products
// each, 18 for the group against 36 for the schoolbook form):
//   lanes 0, 1, 2:  m_i = A_i B_i;
//   lanes 3, 4, 5:  m12 = (A1 + A2)(B1 + B2), m01 = (A0 + A1)(B0 + B1), m02 = (A0 + A2)(B0 + B2);
// and C0 = m0 + t (m12 - m1 - m2), C1 = m01 - m0 - m1 + t m2,
// C2 = m02 - m0 - m2 + m1, C_i = c_i + c_(i+3) t.
struct Fq4 {
    Fq2 r, s;  // r + s t
};
DV_INL Fq4 shfl4(const Fq4& a, int src) { return {shfl2(a.r, src), shfl2(a.s, src)}; }
DV_INL Fq4 add4(const Fq4& a, const Fq4& b) { return {Fq2::add(a.r, b.r), Fq2::add(a.s, b.s)}; }
DV_INL Fq4 sub4(const Fq4& a, const Fq4& b) { return {Fq2::sub(a.r, b.r), Fq2::sub(a.s, b.s)}; }

// Lane k's Karatsuba operand from the group's coefficients: A_k for k < 3,
// the pair sums A1 + A2, A0 + A1, A0 + A2 on lanes 3, 4, 5.  After the
// rotations by 1, 2 and 3 lanes, lane j holds f_j + f_(j+1) and
// f_j + f_(j+2); lanes 3..5 fetch their two halves from lanes (1, 4),
// (0, 3) and (3, 0), each source lane publishing the one sum asked of it.
DV_INL Fq4 k_operand(const Fq2& a, int k, int base) {
    const Fq2 a1 = shfl2(a, base + mod6(k + 1)), a2 = shfl2(a, base + mod6(k + 2));
    const Fq2 a3 = shfl2(a, base + mod6(k + 3));
    const Fq2 s1 = Fq2::add(a, a1), s2 = Fq2::add(a, a2);
    const Fq2 h0 = shfl2(k == 3 ? s2 : s1, base + (k == 3 ? 1 : k == 4 ? 0 : k == 5 ? 3 : k));
    const Fq2 h1 = shfl2(k == 0 ? s2 : s1, base + (k == 3 ? 4 : k == 4 ? 3 : k == 5 ? 0 : k));
    if (k < 3) return {a, a3};
    return k == 5 ? Fq4{h1, h0} : Fq4{h0, h1};
}
// Lane k's coefficient of the product from the six Fq4 products m (one per
// lane): lane i < 3 forms C_i = U + t V from its own m_i, the pair product
// on lane i + 3 and the other two m_j; lane i + 3 takes the t part of C_i.
DV_INL Fq2 k_combine(const Fq4& m, int k, int base) {
    const int i = k < 3 ? k : k - 3;
    const Fq4 q = shfl4(m, base + mod6(k + 3));
    const Fq4 n1 = shfl4(m, base + (i == 2 ? 0 : i + 1));
    const Fq4 n2 = shfl4(m, base + (i == 0 ? 2 : i - 1));
    const Fq4 t = sub4(sub4(q, n1), n2);
    // i = 0: U = m0, V = q - n1 - n2; i = 1: U = q - m1 - n0 = t + n2 - m1 (n2 = m0, n1 = m2),
    // V = n1; i = 2: U = q - m2 - m0 + m1 = t + 2 n2 - m2 (n1 = m0, n2 = m1), V = 0.
    const Fq4 w = i == 1 ? n1 : add4(n2, n2);
    const Fq4 u = i == 0 ? m : sub4(add4(t, w), m);
    const Fq2 vr = i == 0 ? t.r : (i == 1 ? n1.r : Fq2::zero());
    const Fq2 vs = i == 0 ? t.s : (i == 1 ? n1.s : Fq2::zero());
    const Fq2 cr = Fq2::add(u.r, mul_xi(vs)), cs = Fq2::add(u.s, vr);
    const Fq2 hi = shfl2(cs, base + mod6(k + 3));
    return k < 3 ? cr : hi;
}
// x^2 for three Fq2 values, (c0 + c1)(c0 - c1) + 2 c0 c1 u each, the six
// base products in pairs.
DV_INL void fq2_sqr_3(const Fq2* a, Fq2* out) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const Fq::Pair p = Fq::mul2(Fq::add(a[i].c0, a[i].c1), Fq::sub(a[i].c0, a[i].c1), a[i].c0, a[i].c1);
        out[i] = {p.r0, Fq::dbl(p.r1)};
    }
}
// c = a b.
__device__ __noinline__ Fq2 g_mul(const Fq2& a, const Fq2& b, int k, int base) {
    const Fq4 x = k_operand(a, k, base), y = k_operand(b, k, base);
    const Fq2 xs[3] = {x.r, x.s, Fq2::add(x.r, x.s)}, ys[3] = {y.r, y.s, Fq2::add(y.r, y.s)};
    Fq2 p[3];
    fq2_mul_n<3>(xs, ys, p);
    return k_combine({Fq2::add(p[0], mul_xi(p[1])), Fq2::sub(Fq2::sub(p[2], p[0]), p[1])}, k, base);
}
// c = a^2 (the same Karatsuba with Fq4 squares: three Fq2 squares a lane).
__device__ __noinline__ Fq2 g_sqr(const Fq2& a, int k, int base) {
    const Fq4 x = k_operand(a, k, base);
    const Fq2 xs[3] = {x.r, x.s, Fq2::add(x.r, x.s)};
    Fq2 p[3];
    fq2_sqr_3(xs, p);
    return k_combine({Fq2::add(p[0], mul_xi(p[1])), Fq2::sub(Fq2::sub(p[2], p[0]), p[1])}, k, base);
}
// Square of an element of the cyclotomic subgroup (every value after the
// easy part of the final exponentiation), by Granger and Scott ("Faster
// squaring in the cyclotomic subgroup of sixth degree extensions", PKC
// 2010): with A_i = f_i + f_(i+3) t over Fq4 = Fq2[t]/(t^2 - xi), t = w^3,
//   f^2 = (3 A0^2 - 2 conj A0) + (3 t A2^2 + 2 conj A1) w + (3 A1^2 - 2 conj A2) w^2.
// Lane j < 3 squares a_j = f_j and b_j = f_(j+3), lane j + 3 squares
// a_j + b_j; A^2 = (a^2 + xi b^2) + ((a + b)^2 - a^2 - b^2) t.
__device__ __noinline__ Fq2 g_cyc_sqr(const Fq2& f, int k, int base) {
    const int j = k < 3 ? k : k - 3;
    const Fq2 a = shfl2(f, base + j), b = shfl2(f, base + j + 3);
    const Fq2 u = k < 3 ? a : Fq2::add(a, b), v = k < 3 ? b : u;
    // u^2, v^2: (c0 + c1)(c0 - c1) and c0 c1 of each, four base products in two pairs
    const Fq::Pair p0 = Fq::mul2(Fq::add(u.c0, u.c1), Fq::sub(u.c0, u.c1), Fq::add(v.c0, v.c1), Fq::sub(v.c0, v.c1));
    const Fq::Pair p1 = Fq::mul2(u.c0, u.c1, v.c0, v.c1);
    const Fq2 x = {p0.r0, Fq::dbl(p1.r0)}, y = {p0.r1, Fq::dbl(p1.r1)};
    Fq2 sa[3], sb[3], sab[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        sa[m] = shfl2(x, base + m);
        sb[m] = shfl2(y, base + m);
        sab[m] = shfl2(x, base + 3 + m);
    }
    // m = index of the A whose square lane k needs; real part S, t part P
    const int m = k == 0 || k == 3 ? 0 : (k == 2 || k == 5 ? 1 : 2);
    const Fq2 sq_a = m == 0 ? sa[0] : (m == 1 ? sa[1] : sa[2]);
    const Fq2 sq_b = m == 0 ? sb[0] : (m == 1 ? sb[1] : sb[2]);
    const Fq2 sq_ab = m == 0 ? sab[0] : (m == 1 ? sab[1] : sab[2]);
    const Fq2 sr = Fq2::add(sq_a, mul_xi(sq_b));
    const Fq2 pt = Fq2::sub(Fq2::sub(sq_ab, sq_a), sq_b);
    // k = 0: 3 S0 - 2 f0; 3: 3 P0 + 2 f3; 2: 3 S1 - 2 f2; 5: 3 P1 + 2 f5; 4: 3 S2 - 2 f4; 1: 3 xi P2 + 2 f1
    const Fq2 term = k == 0 || k == 2 || k == 4 ? sr : (k == 1 ? mul_xi(pt) : pt);
    const Fq2 t3 = Fq2::add(Fq2::dbl(term), term), f2 = Fq2::dbl(f);
    return k == 0 || k == 2 || k == 4 ? Fq2::sub(t3, f2) : Fq2::add(t3, f2);
}
// f (l0 + l1 w + l3 w^3).
__device__ __noinline__ Fq2 g_mul_line(const Fq2& f, const Fq2& l0, const Fq2& l1, const Fq2& l3, int k, int base) {
    const Fq2 x[3] = {f, shfl2(f, base + mod6(k - 1)), shfl2(f, base + mod6(k - 3))};
    const Fq2 y[3] = {l0, l1, l3};
    Fq2 p[3];
    fq2_mul_n<3>(x, y, p);
    return Fq2::add(Fq2::add(p[0], k < 1 ? mul_xi(p[1]) : p[1]), k < 3 ? mul_xi(p[2]) : p[2]);
}
// f^(q^6): w -> -w.
DV_INL Fq2 g_conj(const Fq2& f, int k) { return (k & 1) ? Fq2::neg(f) : f; }
// q^e-power Frobenius, e = 1, 2, 3.
DV_INL Fq2 g_frob(const Fq2& f, int k, int e) {
    if (e == 2) return Fq2::mul_fq(f, frob2(k));
    Fq2 g = frob1(k);
    if (e == 3) g = Fq2::mul_fq(g, frob2(k));
    return Fq2::mul(Fq2::conj(f), g);
}
// f^-1 = conj(f) / N, N = f conj(f) in Fq6 (the even lanes, v = w^2).
__device__ __noinline__ Fq2 g_inv(const Fq2& f, int k, int base) {
    const Fq2 c = g_conj(f, k);
    const Fq2 n = g_mul(f, c, k, base);
    const Fq6 nn = {shfl2(n, base), shfl2(n, base + 2), shfl2(n, base + 4)};
    const Fq6 ni = f6_inv(nn);
    const Fq2 mine = (k & 1) ? Fq2::zero() : (k == 0 ? ni.c0 : (k == 2 ? ni.c1 : ni.c2));
    return g_mul(c, mine, k, base);
}
// a^z for a in the cyclotomic subgroup (a^-1 = conj a), z the BN seed, over
// its width-4 NAF: a, a^3, a^5, a^7 first (one square, three products), then
// 62 squares and 13 products.
__device__ __noinline__ Fq2 g_pow_z(const Fq2& a, int k, int base) {
    Fq2 tab[4];
    tab[0] = a;
    const Fq2 a2 = g_cyc_sqr(a, k, base);
#pragma unroll 1
    for (int j = 1; j < 4; ++j) tab[j] = g_mul(tab[j - 1], a2, k, base);
    Fq2 r = tab[WNAF_Z[0] >> 1];
#pragma unroll 1
    for (int i = 1; i < WNAF_Z_LEN; ++i) {
        r = g_cyc_sqr(r, k, base);
        const int d = WNAF_Z[i];
        if (d) {
            const Fq2 t = tab[(d < 0 ? -d : d) >> 1];
            r = g_mul(r, d > 0 ? t : g_conj(t, k), k, base);
        }
    }
    return r;
}
DV_INL Fq2 g_one(int k) { return k == 0 ? Fq2::one() : Fq2::zero(); }

struct Tw {
    Fq2 x, y, z;  // Jacobian on the twist
};

// a b with the two base products a0 b0, a1 b1 issued as a pair.
DV_INL Fq2 fq2_mul_fast(const Fq2& a, const Fq2& b) {
    const Fq::Pair p = Fq::mul2(a.c0, b.c0, a.c1, b.c1);
    const Fq t = Fq::mul(Fq::add(a.c0, a.c1), Fq::add(b.c0, b.c1));
    return {Fq::sub(p.r0, p.r1), Fq::sub(Fq::sub(t, p.r0), p.r1)};
}
DV_INL Fq2 pick(int k, const Fq2& v0, const Fq2& v1, const Fq2& v2, const Fq2& v3, const Fq2& v4, const Fq2& v5) {
    return k == 0 ? v0 : k == 1 ? v1 : k == 2 ? v2 : k == 3 ? v3 : k == 4 ? v4 : v5;
}
// Each lane of the group computes one Fq2 product, its operands chosen by
// k, and gets every lane's product back.
DV_INL void level(const Fq2& a, const Fq2& b, int base, Fq2* out, int n) {
    Fq2 p;
    fq2_mul_n<1>(&a, &b, &p);
#pragma unroll
    for (int j = 0; j < 6; ++j)
        if (j < n) out[j] = shfl2(p, base + j);
}
DV_INL Fq2 fq2_of(const Fq& x) { return {x, Fq::zero()}; }

// T <- 2T and the line's (w^0, w^1, w^3) terms at P, the products spread
// over the group in three dependency levels:
//   A = X^2, B = Y^2, ZZ = Z^2, YZ = Y Z;
//   C = B^2, S = (X + B)^2, E ZZ, Z3 ZZ, E X, E^2   (E = 3A, Z3 = 2 Y Z);
//   E (D - X3), Z3 ZZ yp, E ZZ xp                   (D = 2(S - A - C), X3 = E^2 - 2D).
__device__ __noinline__ void dbl_step(Tw& t, const Fq& xp, const Fq& yp, Fq2& l0, Fq2& l1, Fq2& l3, int k, int base) {
    Fq2 v[6];
    level(pick(k, t.x, t.y, t.z, t.y, t.x, t.x), pick(k, t.x, t.y, t.z, t.z, t.x, t.x), base, v, 4);
    const Fq2 a = v[0], b = v[1], zz = v[2];
    const Fq2 e = Fq2::add(Fq2::dbl(a), a), z3 = Fq2::dbl(v[3]), xb = Fq2::add(t.x, b);
    level(pick(k, b, xb, e, z3, e, e), pick(k, b, xb, zz, zz, t.x, e), base, v, 6);
    const Fq2 c = v[0], ezz = v[2], z3zz = v[3], ex = v[4];
    const Fq2 d = Fq2::dbl(Fq2::sub(Fq2::sub(v[1], a), c));
    const Fq2 x3 = Fq2::sub(v[5], Fq2::dbl(d));
    level(pick(k, e, z3zz, ezz, e, e, e), pick(k, Fq2::sub(d, x3), fq2_of(yp), fq2_of(xp), e, e, e), base, v, 3);
    l0 = v[1];
    l1 = Fq2::neg(v[2]);
    l3 = Fq2::sub(ex, Fq2::dbl(b));
    t.y = Fq2::sub(v[0], Fq2::dbl(Fq2::dbl(Fq2::dbl(c))));
    t.x = x3;
    t.z = z3;
}
// T <- T + S (S affine) and the line at P, in five levels:
//   ZZ = Z^2 (every lane); U2 = xs ZZ, ZZZ = Z ZZ;
//   S2 = ys ZZZ, HH = H^2, (Z + H)^2              (H = U2 - X);
//   J = H I, V = X I, r^2, r xs, r xp, Z3 ys      (I = 4 HH, r = 2(S2 - Y), Z3 = (Z + H)^2 - ZZ - HH);
//   r (V - X3), Y J, Z3 yp                        (X3 = r^2 - J - 2V).
__device__ __noinline__ void add_step(Tw& t, const Fq2& xs, const Fq2& ys, const Fq& xp, const Fq& yp, Fq2& l0,
                                      Fq2& l1, Fq2& l3, int k, int base) {
    Fq2 v[6];
    const Fq2 zz = fq2_mul_fast(t.z, t.z);
    level(pick(k, xs, t.z, xs, xs, xs, xs), pick(k, zz, zz, zz, zz, zz, zz), base, v, 2);
    const Fq2 h = Fq2::sub(v[0], t.x), zh = Fq2::add(t.z, h);
    level(pick(k, ys, h, zh, h, h, h), pick(k, v[1], h, zh, h, h, h), base, v, 3);
    const Fq2 hh = v[1];
    const Fq2 i = Fq2::dbl(Fq2::dbl(hh));
    const Fq2 r = Fq2::dbl(Fq2::sub(v[0], t.y));
    const Fq2 z3 = Fq2::sub(Fq2::sub(v[2], zz), hh);
    level(pick(k, h, t.x, r, r, r, z3), pick(k, i, i, r, xs, fq2_of(xp), ys), base, v, 6);
    const Fq2 j = v[0], vv = v[1], rxs = v[3], rxp = v[4], z3ys = v[5];
    const Fq2 x3 = Fq2::sub(Fq2::sub(v[2], j), Fq2::dbl(vv));
    level(pick(k, r, t.y, z3, r, r, r), pick(k, Fq2::sub(vv, x3), j, fq2_of(yp), r, r, r), base, v, 3);
    l0 = v[2];
    l1 = Fq2::neg(rxp);
    l3 = Fq2::sub(rxs, z3ys);
    t.y = Fq2::sub(v[0], Fq2::dbl(v[1]));
    t.x = x3;
    t.z = z3;
}

struct GroupLane {
    int k, base;
    uint64_t group;  // global group index
    bool live;       // lanes 0..29 of the warp
};
DV_INL GroupLane group_lane() {
    const int l = threadIdx.x & 31;
    const int k = l < GL * GROUPS_PER_WARP ? l % GL : l - GL * GROUPS_PER_WARP;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    return {k, l - k, warp * GROUPS_PER_WARP + (uint64_t)(l / GL), l < GL * GROUPS_PER_WARP};
}

// ------------------------------------------------------------------ prepared G2 points
// A line of the Miller loop at P = (xp, yp) is A yp + (B xp) w + C w^3 with
// A, B, C depending on Q alone (the doubling: A = 2 Y Z^3, B = -3 X^2 Z^2,
// C = 3 X^3 - 2 Y^2; the addition: A = 2 Z H, B = -2 R, C = 2 R xs - 2 Z H ys).
// Preparing Q records the LINES triples of its loop once -- arkworks'
// G2Prepared, which the reference caches per distinct G2 point
// (crates/protocol/src/verification.rs:105-126) -- so the loop of every term
// that shares Q only scales them by its P and multiplies them in.
struct __align__(16) Line {
    Fq2 a, b, c;
};
constexpr int LINES = 88;  // 65 doublings, 21 NAF additions (nonzero digits after the first), 2 Frobenius additions

// The doubling and addition steps without P: the same levels, minus the
// products by xp and yp.
__device__ __noinline__ void prep_dbl(Tw& t, Line& l, int k, int base) {
    Fq2 v[6];
    level(pick(k, t.x, t.y, t.z, t.y, t.x, t.x), pick(k, t.x, t.y, t.z, t.z, t.x, t.x), base, v, 4);
    const Fq2 a = v[0], b = v[1], zz = v[2];
    const Fq2 e = Fq2::add(Fq2::dbl(a), a), z3 = Fq2::dbl(v[3]), xb = Fq2::add(t.x, b);
    level(pick(k, b, xb, e, z3, e, e), pick(k, b, xb, zz, zz, t.x, e), base, v, 6);
    const Fq2 c = v[0], ezz = v[2], z3zz = v[3], ex = v[4];
    const Fq2 d = Fq2::dbl(Fq2::sub(Fq2::sub(v[1], a), c));
    const Fq2 x3 = Fq2::sub(v[5], Fq2::dbl(d));
    level(e, Fq2::sub(d, x3), base, v, 1);
    l = {z3zz, Fq2::neg(ezz), Fq2::sub(ex, Fq2::dbl(b))};
    t.y = Fq2::sub(v[0], Fq2::dbl(Fq2::dbl(Fq2::dbl(c))));
    t.x = x3;
    t.z = z3;
}
__device__ __noinline__ void prep_add(Tw& t, const Fq2& xs, const Fq2& ys, Line& l, int k, int base) {
    Fq2 v[6];
    const Fq2 zz = fq2_mul_fast(t.z, t.z);
    level(pick(k, xs, t.z, xs, xs, xs, xs), pick(k, zz, zz, zz, zz, zz, zz), base, v, 2);
    const Fq2 h = Fq2::sub(v[0], t.x), zh = Fq2::add(t.z, h);
    level(pick(k, ys, h, zh, h, h, h), pick(k, v[1], h, zh, h, h, h), base, v, 3);
    const Fq2 hh = v[1];
    const Fq2 i = Fq2::dbl(Fq2::dbl(hh));
    const Fq2 r = Fq2::dbl(Fq2::sub(v[0], t.y));
    const Fq2 z3 = Fq2::sub(Fq2::sub(v[2], zz), hh);
    level(pick(k, h, t.x, r, r, z3, r), pick(k, i, i, r, xs, ys, r), base, v, 5);
    const Fq2 j = v[0], vv = v[1], rxs = v[3], z3ys = v[4];
    const Fq2 x3 = Fq2::sub(Fq2::sub(v[2], j), Fq2::dbl(vv));
    level(pick(k, r, t.y, r, r, r, r), pick(k, Fq2::sub(vv, x3), j, r, r, r, r), base, v, 2);
    l = {z3, Fq2::neg(r), Fq2::sub(rxs, z3ys)};
    t.y = Fq2::sub(v[0], Fq2::dbl(v[1]));
    t.x = x3;
    t.z = z3;
}

// The LINES triples of every Q (one lane group each) at lines[LINES q ..],
// and inf[q] = 1 for Q at infinity (whose lines count as 1).
__global__ void __launch_bounds__(128) k_prepare(const G2A* __restrict__ g2, uint64_t nq, Line* __restrict__ lines,
                                                 uint32_t* __restrict__ inf) {
    const GroupLane g = group_lane();
    const bool mine = g.live && g.group < nq;
    const uint64_t qi = mine ? g.group : 0;
    const G2A q = g2[qi];
    if (mine && g.k == 0) inf[qi] = q.is_inf() ? 1u : 0u;
    Line* out = lines + (uint64_t)LINES * qi;
    Tw t{q.x, q.y, Fq2::one()};
    Line l;
    int n = 0;
    const Fq2 nqy = Fq2::neg(q.y);
    auto put = [&](const Line& x) {
        if (mine && g.k < 3) (&out[n].a)[g.k] = (&x.a)[g.k];
        ++n;
    };
    for (int i = 1; i < NAF_LEN; ++i) {
        prep_dbl(t, l, g.k, g.base);
        put(l);
        const int d = NAF_6Z2[i];
        if (d) {
            prep_add(t, q.x, d > 0 ? q.y : nqy, l, g.k, g.base);
            put(l);
        }
    }
    const Fq2 x1 = Fq2::mul(Fq2::conj(q.x), frob1(2)), y1 = Fq2::mul(Fq2::conj(q.y), frob1(3));
    const Fq2 x2 = Fq2::mul_fq(q.x, frob2(2)), y2 = Fq2::neg(Fq2::mul_fq(q.y, frob2(3)));
    prep_add(t, x1, y1, l, g.k, g.base);
    put(l);
    prep_add(t, x2, y2, l, g.k, g.base);
    put(l);
}

// A line A yp + (B xp) w + C w^3 scaled to its P: coefficients of w^0,
// w^1, w^3.  A term with P or Q at infinity, or past its equation's count,
// takes the line 1.
struct SLine {
    Fq2 l0, l1, l3;
};
DV_INL SLine line_one() { return {Fq2::one(), Fq2::zero(), Fq2::zero()}; }
// One term's scaling: the four base products A yp, B xp one per lane
// (lanes 0..3), shared by shuffles.
DV_INL SLine scale_one(const Line& x, const G1A& p, bool one, int k, int base) {
    const Fq u = k == 0 ? x.a.c0 : k == 1 ? x.a.c1 : k == 2 ? x.b.c0 : x.b.c1;
    const Fq r = Fq::mul(u, k < 2 ? p.y : p.x);
    const SLine l = {{shfl_fq(r, base), shfl_fq(r, base + 1)}, {shfl_fq(r, base + 2), shfl_fq(r, base + 3)}, x.c};
    return one ? line_one() : l;
}
// Two terms' scaling: eight base products, lane k forms product k and lanes
// 0, 1 also products 6, 7 (x: A yp, B xp of the first term, then of the
// second).
DV_INL void scale_two(const Line& x, const G1A& p, bool one_x, const Line& y, const G1A& q, bool one_y, int k,
                      int base, SLine& a, SLine& b) {
    const Fq u0 = k == 0 ? x.a.c0 : k == 1 ? x.a.c1 : k == 2 ? x.b.c0 : k == 3 ? x.b.c1 : k == 4 ? y.a.c0 : y.a.c1;
    const Fq v0 = k < 2 ? p.y : (k < 4 ? p.x : q.y);
    const Fq::Pair r = Fq::mul2(u0, v0, k == 0 ? y.b.c0 : y.b.c1, q.x);
    const SLine la = {{shfl_fq(r.r0, base), shfl_fq(r.r0, base + 1)}, {shfl_fq(r.r0, base + 2), shfl_fq(r.r0, base + 3)},
                      x.c};
    const SLine lb = {{shfl_fq(r.r0, base + 4), shfl_fq(r.r0, base + 5)}, {shfl_fq(r.r1, base), shfl_fq(r.r1, base + 1)},
                      y.c};
    a = one_x ? line_one() : la;
    b = one_y ? line_one() : lb;
}
// (a0 + a1 w + a3 w^3)(b0 + b1 w + b3 w^3): the Karatsuba products p0 = a0 b0,
// p1 = a1 b1, p2 = a3 b3, p3 = (a0 + a1)(b0 + b1), p4 = (a0 + a3)(b0 + b3),
// p5 = (a1 + a3)(b1 + b3), one per lane; c0 = p0 + xi p2, c1 = p3 - p0 - p1,
// c2 = p1, c3 = p4 - p0 - p2, c4 = p5 - p1 - p2, c5 = 0.
__device__ __noinline__ Fq2 g_line_line(const SLine& a, const SLine& b, int k, int base) {
    const Fq2 x = k == 0 ? a.l0 : k == 1 ? a.l1 : k == 2 ? a.l3 : Fq2::add(k == 5 ? a.l1 : a.l0, k == 3 ? a.l1 : a.l3);
    const Fq2 y = k == 0 ? b.l0 : k == 1 ? b.l1 : k == 2 ? b.l3 : Fq2::add(k == 5 ? b.l1 : b.l0, k == 3 ? b.l1 : b.l3);
    Fq2 p;
    fq2_mul_n<1>(&x, &y, &p);
    const Fq2 m = shfl2(p, base + (k == 1 ? 3 : k == 2 ? 1 : k == 3 ? 4 : k == 4 ? 5 : 0));
    const Fq2 p0 = shfl2(p, base), p1 = shfl2(p, base + 1), p2 = shfl2(p, base + 2);
    const Fq2 d = Fq2::sub(Fq2::sub(m, k == 4 ? p1 : p0), k == 1 ? p1 : p2);
    return k == 0 ? Fq2::add(p0, mul_xi(p2)) : k == 2 ? m : k == 5 ? Fq2::zero() : d;
}

// Miller value of every equation from its terms' P and prepared Q, one lane
// group per equation and one f for all its terms (the multi-Miller loop):
// every step squares f once and multiplies in the lines of all the terms,
// two terms' lines first multiplied together (six Fq2 products, one per
// lane) and then into f by one product, a last odd term by the sparse line
// product.  Every group of a warp runs the warp's largest term count.
// Value of equation e at out[6 e + k]; without offsets every term is its own
// equation (a group per term, for batches too small to fill the GPU, whose
// terms then meet in the final exponentiation).
__global__ void __launch_bounds__(128) k_miller_multi(const G1A* __restrict__ g1, const uint32_t* __restrict__ qidx,
                                                      const uint32_t* __restrict__ qinf,
                                                      const Line* __restrict__ lines,
                                                      const uint64_t* __restrict__ offsets, uint64_t equations,
                                                      Fq2* __restrict__ out) {
    const GroupLane g = group_lane();
    const bool mine = g.live && g.group < equations;
    const uint64_t e = mine ? g.group : 0;
    const uint64_t first = !mine ? 0 : offsets ? offsets[e] : e;
    const uint64_t count = !mine ? 0 : offsets ? offsets[e + 1] - first : 1;
    uint64_t most = count;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const uint64_t o = __shfl_xor_sync(FULL, most, off);
        most = o > most ? o : most;
    }
    // term j of this group at line n (term 0 of the call stands in past the
    // group's count, which is then nonzero somewhere in the warp); true when
    // its line counts as 1
    auto term = [&](uint64_t j, int n, G1A& p, Line& l) {
        const bool have = j < count;
        const uint64_t t = have ? first + j : 0;
        p = g1[t];
        const uint32_t qi = qidx[t];
        l = lines[(uint64_t)LINES * qi + n];
        return !have || p.is_inf() || qinf[qi] != 0;
    };
    Fq2 f = g_one(g.k);
    auto apply = [&](int n) {
        for (uint64_t j = 0; j < most; j += 2) {
            G1A pa, pb;
            Line la, lb;
            const bool oa = term(j, n, pa, la);
            if (j + 1 < most) {
                const bool ob = term(j + 1, n, pb, lb);
                SLine a, b;
                scale_two(la, pa, oa, lb, pb, ob, g.k, g.base, a, b);
                f = g_mul(f, g_line_line(a, b, g.k, g.base), g.k, g.base);
            } else {
                const SLine a = scale_one(la, pa, oa, g.k, g.base);
                f = g_mul_line(f, a.l0, a.l1, a.l3, g.k, g.base);
            }
        }
    };
    int n = 0;
    for (int i = 1; i < NAF_LEN; ++i) {
        if (i > 1) f = g_sqr(f, g.k, g.base);
        apply(n++);
        if (NAF_6Z2[i]) apply(n++);
    }
    apply(n++);
    apply(n++);
    if (mine) out[6 * e + g.k] = f;
}

// Miller value of (P, Q) as this lane's coefficient; every lane holds T and
// the lines (their products are spread over the group).
__device__ Fq2 g_miller(const G1A& p, const G2A& q, int k, int base) {
    Tw t{q.x, q.y, Fq2::one()};
    Fq2 f = g_one(k);
    Fq2 l0, l1, l3;
    const Fq2 nqy = Fq2::neg(q.y);
    for (int i = 1; i < NAF_LEN; ++i) {
        dbl_step(t, p.x, p.y, l0, l1, l3, k, base);
        f = g_mul_line(g_sqr(f, k, base), l0, l1, l3, k, base);
        const int d = NAF_6Z2[i];
        if (d) {
            add_step(t, q.x, d > 0 ? q.y : nqy, p.x, p.y, l0, l1, l3, k, base);
            f = g_mul_line(f, l0, l1, l3, k, base);
        }
    }
    // pi(Q) = (conj(x) xi^((q-1)/3), conj(y) xi^((q-1)/2)); -pi^2(Q) = (x xi^((q^2-1)/3), -y xi^((q^2-1)/2))
    const Fq2 x1 = Fq2::mul(Fq2::conj(q.x), frob1(2)), y1 = Fq2::mul(Fq2::conj(q.y), frob1(3));
    const Fq2 x2 = Fq2::mul_fq(q.x, frob2(2)), y2 = Fq2::neg(Fq2::mul_fq(q.y, frob2(3)));
    add_step(t, x1, y1, p.x, p.y, l0, l1, l3, k, base);
    f = g_mul_line(f, l0, l1, l3, k, base);
    add_step(t, x2, y2, p.x, p.y, l0, l1, l3, k, base);
    return g_mul_line(f, l0, l1, l3, k, base);
}

__device__ Fq2 g_final_exponentiation(const Fq2& m, int k, int base) {
    Fq2 f = g_mul(g_conj(m, k), g_inv(m, k, base), k, base);  // ^(q^6 - 1)
    f = g_mul(g_frob(f, k, 2), f, k, base);                    // ^(q^2 + 1)
    const Fq2 a = g_pow_z(f, k, base);
    const Fq2 b = g_pow_z(a, k, base);
    const Fq2 c = g_pow_z(b, k, base);
    const Fq2 a2 = g_cyc_sqr(a, k, base), a4 = g_cyc_sqr(a2, k, base), a6 = g_mul(a4, a2, k, base);
    const Fq2 b2 = g_cyc_sqr(b, k, base), b6 = g_mul(g_cyc_sqr(b2, k, base), b2, k, base);
    const Fq2 b12 = g_cyc_sqr(b6, k, base);
    const Fq2 c4 = g_cyc_sqr(g_cyc_sqr(c, k, base), k, base), c12 = g_mul(g_cyc_sqr(c4, k, base), c4, k, base);
    const Fq2 tt = g_mul(c12, b6, k, base);
    const Fq2 l1 = g_mul(tt, a4, k, base);
    const Fq2 l2 = g_mul(tt, a6, k, base);
    const Fq2 l3 = g_mul(l1, g_conj(f, k), k, base);
    const Fq2 l0 = g_mul(g_mul(g_mul(c12, b12, k, base), a6, k, base), f, k, base);
    Fq2 r = g_mul(l0, g_frob(l1, k, 1), k, base);
    r = g_mul(r, g_frob(l2, k, 2), k, base);
    return g_mul(r, g_frob(l3, k, 3), k, base);
}

// Miller value of every term, one lane group per term (coefficient k of
// term t at out[6 t + k]); infinity on either side gives one.
__global__ void __launch_bounds__(128) k_miller(const G1A* __restrict__ g1, const G2A* __restrict__ g2,
                                                uint64_t terms, Fq2* __restrict__ out) {
    const GroupLane g = group_lane();
    const bool mine = g.live && g.group < terms;
    const uint64_t t = mine ? g.group : 0;  // idle lanes compute on term 0
    const G1A p = g1[t];
    const G2A q = g2[t];
    const Fq2 f = g_miller(p, q, g.k, g.base);
    if (mine) out[6 * t + g.k] = (p.is_inf() || q.is_inf()) ? g_one(g.k) : f;
}

// One lane group per equation: product of its terms' values (every group of
// a warp runs the warp's largest term count, multiplying by one past its
// own; without offsets one value per equation), final exponentiation,
// verdict, and with gt the canonical GT element.
__global__ void __launch_bounds__(128) k_final_exp(const Fq2* __restrict__ miller, const uint64_t* __restrict__ offsets,
                                                   uint64_t equations, uint8_t* __restrict__ verdicts,
                                                   uint8_t* __restrict__ gt) {
    const GroupLane g = group_lane();
    const bool mine = g.live && g.group < equations;
    const uint64_t e = mine ? g.group : 0;
    const uint64_t first = !mine ? 0 : offsets ? offsets[e] : e;
    const uint64_t count = !mine ? 0 : offsets ? offsets[e + 1] - first : 1;
    uint64_t most = count;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const uint64_t o = __shfl_xor_sync(FULL, most, off);
        most = o > most ? o : most;
    }
    Fq2 f = g_one(g.k);
    for (uint64_t t = 0; t < most; ++t) {
        const Fq2 v = t < count ? miller[6 * (first + t) + g.k] : g_one(g.k);
        f = t == 0 ? v : g_mul(f, v, g.k, g.base);
    }
    const Fq2 r = g_final_exponentiation(f, g.k, g.base);
    const bool coef_ok = g.k == 0 ? (r.c0 == Fq::one() && r.c1.is_zero()) : r.is_zero();
    const unsigned ok = __ballot_sync(FULL, coef_ok);
    if (!mine) return;
    if (verdicts && g.k == 0) verdicts[e] = ((ok >> g.base) & 0x3fu) == 0x3fu ? 1 : 0;
    if (gt) {
        // tower order: w^0, w^2, w^4, w^1, w^3, w^5
        const int slot = (g.k & 1) ? 3 + (g.k >> 1) : (g.k >> 1);
        store_canonical(gt + 384 * e + 64 * slot, r.c0);
        store_canonical(gt + 384 * e + 64 * slot + 32, r.c1);
    }
}

constexpr uint64_t PREP_MAX = 1ull << 17;  // distinct G2 points prepared in one call (17.5 KB each)

constexpr uint64_t GROUPS_PER_BLOCK = 128 / 32 * GROUPS_PER_WARP;

unsigned group_blocks(uint64_t groups) { return (unsigned)((groups + GROUPS_PER_BLOCK - 1) / GROUPS_PER_BLOCK); }

// Whether the prepared Miller loops run one group per equation (the
// multi-Miller loop, fewer instructions) rather than one per term (shorter
// chains): per equation once a group per term would take more than one wave
// of resident blocks (on B200, 2 blocks of 20 groups per SM: 5920 terms).
bool miller_per_equation(uint64_t terms) {
    static const uint64_t wave = [] {
        int blocks = 0;
        DV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_miller_multi, 128, 0));
        return (uint64_t)sm_count() * (uint64_t)std::max(1, blocks) * GROUPS_PER_BLOCK;
    }();
    return terms > wave;
}

// 128-byte G2 wire points as hash keys (FNV-1a over the words).
struct G2Key {
    uint64_t w[16];
    bool operator==(const G2Key& o) const { return memcmp(w, o.w, sizeof(w)) == 0; }
};
struct G2KeyHash {
    size_t operator()(const G2Key& k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint64_t x : k.w) h = (h ^ x) * 1099511628211ull;
        return (size_t)h;
    }
};

// Device copy of the equations' term offsets.
uint64_t* upload_offsets(Backend& b, const uint64_t* offsets, uint64_t equations, cudaStream_t st) {
    uint64_t* d_off = b.idx.as<uint64_t>(equations + 1);
    DV_CUDA(cudaMemcpyAsync(d_off, offsets, 8 * (equations + 1), cudaMemcpyHostToDevice, st));
    return d_off;
}

// Final exponentiation of the Miller values in mil (one per term, folded per
// equation by the device offsets d_off; one per equation when d_off is
// null), verdicts / GT elements back to the host.
void finish_equations(Backend& b, Fq2* mil, const uint64_t* d_off, uint64_t equations, uint8_t* verdicts,
                      uint8_t* gt, const uint32_t* bad, const std::vector<uint64_t>* g2_first, cudaStream_t st) {
    // GT elements first (16-byte aligned stores), then the verdict bytes
    uint8_t* d_gt = b.out_buf.as<uint8_t>(equations * ((gt ? 384 : 0) + 1));
    uint8_t* d_out = d_gt + (gt ? 384 * equations : 0);
    k_final_exp<<<group_blocks(equations), 128, 0, st>>>(mil, d_off, equations, d_out, gt ? d_gt : nullptr);
    DV_LAUNCH();
    uint32_t hbad[2];
    DV_CUDA(cudaMemcpyAsync(hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (hbad[0] != 0xffffffffu) throw InvalidArgument("invalid G1 point at term " + std::to_string(hbad[0]));
    if (hbad[1] != 0xffffffffu)
        throw InvalidArgument("invalid G2 point at term " +
                              std::to_string(g2_first ? (*g2_first)[hbad[1]] : (uint64_t)hbad[1]));
    if (verdicts) DV_CUDA(cudaMemcpy(verdicts, d_out, equations, cudaMemcpyDeviceToHost));
    if (gt) DV_CUDA(cudaMemcpy(gt, d_gt, 384 * equations, cudaMemcpyDeviceToHost));
}

}  // namespace

struct PreparedG2 {
    uint64_t n = 0;
    DevBuf points;  // G2A (Montgomery affine)
    DevBuf lines;   // LINES per point
    DevBuf inf;     // u32 per point: 1 at infinity
};
struct PairingState {
    std::map<uint64_t, std::unique_ptr<PreparedG2>> prepared;
    DevBuf lines, inf, qidx;
};

namespace {

PairingState& pairing_state(Backend& b) {
    if (!b.pairing) b.pairing = std::make_shared<PairingState>();
    return *b.pairing;
}

void pairing_run(Backend& b, const uint8_t* g1, const uint8_t* g2, uint64_t terms, const uint64_t* offsets,
                 uint64_t equations, uint8_t* verdicts, uint8_t* gt, cudaStream_t st) {
    // the distinct G2 points of the call: shared ones are prepared once
    std::vector<uint32_t> qidx;
    std::vector<uint64_t> first;
    std::vector<uint8_t> distinct;
    if (terms > 1) {
        std::unordered_map<G2Key, uint32_t, G2KeyHash> seen;
        seen.reserve(terms);
        qidx.resize(terms);
        for (uint64_t t = 0; t < terms; ++t) {
            G2Key key;
            memcpy(key.w, g2 + 128 * t, 128);
            const auto it = seen.emplace(key, (uint32_t)first.size());
            if (it.second) {
                first.push_back(t);
                distinct.insert(distinct.end(), g2 + 128 * t, g2 + 128 * (t + 1));
            }
            qidx[t] = it.first->second;
        }
    }
    const uint64_t nq = first.size();
    const bool prepared = terms > 1 && nq < terms && nq <= PREP_MAX;
    const bool multi = prepared && miller_per_equation(terms);
    const uint64_t g2_count = prepared ? nq : terms;
    uint8_t* d_in = b.in_points.as<uint8_t>(64 * terms + 128 * g2_count);
    DV_CUDA(cudaMemcpyAsync(d_in, g1, 64 * terms, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(d_in + 64 * terms, prepared ? distinct.data() : g2, 128 * g2_count,
                            cudaMemcpyHostToDevice, st));
    G1A* p = b.conv_points.as<G1A>(terms + 2 * g2_count);  // G1A (64 B) then G2A (128 B)
    G2A* q = reinterpret_cast<G2A*>(p + terms);
    uint32_t* bad = b.err.as<uint32_t>(2);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, 2 * sizeof(uint32_t), st));
    convert_points<Fq>(d_in, p, terms, bad, st);
    convert_points<Fq2>(d_in + 64 * terms, q, g2_count, bad + 1, st);
    uint64_t* d_off = upload_offsets(b, offsets, equations, st);
    Fq2* mil = b.aux.as<Fq2>(6 * std::max<uint64_t>(1, std::max(terms, equations)));
    if (prepared) {
        PairingState& ps = pairing_state(b);
        Line* lines = ps.lines.as<Line>((uint64_t)LINES * nq);
        uint32_t* qinf = ps.inf.as<uint32_t>(nq);
        uint32_t* d_qidx = ps.qidx.as<uint32_t>(terms);
        DV_CUDA(cudaMemcpyAsync(d_qidx, qidx.data(), 4 * terms, cudaMemcpyHostToDevice, st));
        k_prepare<<<group_blocks(nq), 128, 0, st>>>(q, nq, lines, qinf);
        DV_LAUNCH();
        if (multi)
            k_miller_multi<<<group_blocks(equations), 128, 0, st>>>(p, d_qidx, qinf, lines, d_off, equations, mil);
        else
            k_miller_multi<<<group_blocks(terms), 128, 0, st>>>(p, d_qidx, qinf, lines, nullptr, terms, mil);
        DV_LAUNCH();
    } else if (terms) {
        k_miller<<<group_blocks(terms), 128, 0, st>>>(p, q, terms, mil);
        DV_LAUNCH();
    }
    finish_equations(b, mil, prepared && multi ? nullptr : d_off, equations, verdicts, gt, bad,
                     prepared ? &first : nullptr, st);
}

}  // namespace

// Bytes of one prepared G2 point (its Miller loop's line triples).
uint64_t pairing_prepared_bytes() { return (uint64_t)LINES * sizeof(Line); }

// Prepares nq Montgomery affine G2 points of q: their lines into `lines`
// (nq * pairing_prepared_bytes()) and a u32 per point into qinf (1 at
// infinity).  No host synchronisation; the buffers are the caller's, so a
// set of fixed points (a verifying key) can be prepared once and reused.
void pairing_prepare_device(const G2A* q, uint64_t nq, void* lines, uint32_t* qinf, cudaStream_t st) {
    if (!nq) return;
    if (nq > PREP_MAX) throw InvalidArgument("too many distinct G2 points in one check");
    k_prepare<<<group_blocks(nq), 128, 0, st>>>(q, nq, static_cast<Line*>(lines), qinf);
    DV_LAUNCH();
}

// Pairing-product checks over prepared G2 points, with no host
// synchronisation: equation e holds iff prod over terms
// [d_off[e], d_off[e+1]) of e(p[k], Q[d_qidx[k]]) is one, where Q's lines
// and infinity flags are at lines / qinf (pairing_prepare_device);
// d_verdicts[e] = 1 / 0.  p: Montgomery affine G1 terms.  Scratch comes
// from the backend.
void pairing_check_prepared(Backend& b, const G1A* p, uint64_t terms, const void* lines, const uint32_t* qinf,
                            const uint32_t* d_qidx, const uint64_t* d_off, uint64_t equations, uint8_t* d_verdicts,
                            cudaStream_t st) {
    if (!equations) return;
    const Line* ln = static_cast<const Line*>(lines);
    Fq2* mil = b.aux.as<Fq2>(6 * std::max<uint64_t>(1, std::max(terms, equations)));
    const bool multi = miller_per_equation(terms);
    if (multi) {
        k_miller_multi<<<group_blocks(equations), 128, 0, st>>>(p, d_qidx, qinf, ln, d_off, equations, mil);
        DV_LAUNCH();
    } else if (terms) {
        k_miller_multi<<<group_blocks(terms), 128, 0, st>>>(p, d_qidx, qinf, ln, nullptr, terms, mil);
        DV_LAUNCH();
    }
    k_final_exp<<<group_blocks(equations), 128, 0, st>>>(mil, multi ? nullptr : d_off, equations, d_verdicts,
                                                         nullptr);
    DV_LAUNCH();
}

// The same checks with the nq G2 points of q prepared first (into the
// backend's pairing scratch).  For callers that build their equations on
// the device (the Dynaverse verifier, dynaverse.cu).
void pairing_check_device(Backend& b, const G1A* p, uint64_t terms, const G2A* q, uint64_t nq,
                          const uint32_t* d_qidx, const uint64_t* d_off, uint64_t equations, uint8_t* d_verdicts,
                          cudaStream_t st) {
    if (!equations) return;
    if (nq > PREP_MAX) throw InvalidArgument("too many distinct G2 points in one check");
    PairingState& ps = pairing_state(b);
    Line* lines = ps.lines.as<Line>((uint64_t)LINES * std::max<uint64_t>(1, nq));
    uint32_t* qinf = ps.inf.as<uint32_t>(std::max<uint64_t>(1, nq));
    pairing_prepare_device(q, nq, lines, qinf, st);
    pairing_check_prepared(b, p, terms, lines, qinf, d_qidx, d_off, equations, d_verdicts, st);
}

namespace {

void check_offsets(const uint64_t* offsets, size_t equations) {
    require(offsets && equations >= 1 && equations <= (1u << 24), "invalid pairing check arguments");
    require(offsets[0] == 0, "pairing offsets must start at 0");
    for (size_t e = 0; e < equations; ++e) require(offsets[e + 1] >= offsets[e], "pairing offsets must not decrease");
    require(offsets[equations] <= (1u << 24), "invalid pairing terms");
}

}  // namespace
}  // namespace dv

using namespace dv;

extern "C" int dvgpu_bn254_pairing_check(void* opaque, const uint8_t* g1, const uint8_t* g2, const uint64_t* offsets,
                                         size_t equations, uint8_t* verdicts, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        check_offsets(offsets, equations);
        const uint64_t terms = offsets[equations];
        require(verdicts && (g1 || !terms) && (g2 || !terms), "invalid pairing terms");
        pairing_run(b, g1, g2, terms, offsets, equations, verdicts, nullptr, b.stream);
    });
}

extern "C" int dvgpu_bn254_pairing(void* opaque, const uint8_t* g1, const uint8_t* g2, size_t n, uint8_t* gt,
                                   char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(g1 && g2 && gt && n >= 1 && n <= (1u << 24), "invalid pairing arguments");
        std::vector<uint64_t> off(n + 1);
        for (size_t i = 0; i <= n; ++i) off[i] = i;
        pairing_run(b, g1, g2, n, off.data(), n, nullptr, gt, b.stream);
    });
}

extern "C" int dvgpu_bn254_g2_prepare(void* opaque, const uint8_t* g2, size_t n, uint64_t* prepared, char* error,
                                      size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(g2 && prepared && n >= 1 && n <= PREP_MAX, "invalid G2 preparation arguments (1..2^17 points)");
        const cudaStream_t st = b.stream;
        auto pg = std::make_unique<PreparedG2>();
        pg->n = n;
        uint8_t* d_in = b.in_points.as<uint8_t>(128 * n);
        DV_CUDA(cudaMemcpyAsync(d_in, g2, 128 * n, cudaMemcpyHostToDevice, st));
        uint32_t* bad = b.err.as<uint32_t>(1);
        DV_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(uint32_t), st));
        G2A* q = pg->points.as<G2A>(n);
        convert_points<Fq2>(d_in, q, n, bad, st);
        k_prepare<<<group_blocks(n), 128, 0, st>>>(q, n, pg->lines.as<Line>((uint64_t)LINES * n),
                                                   pg->inf.as<uint32_t>(n));
        DV_LAUNCH();
        const uint32_t first_bad = read_err_word(b, bad, st);
        if (first_bad != 0xffffffffu) throw InvalidArgument("invalid G2 point at index " + std::to_string(first_bad));
        const uint64_t h = b.next_handle++;
        pairing_state(b).prepared[h] = std::move(pg);
        *prepared = h;
    });
}

extern "C" int dvgpu_bn254_g2_prepared_release(void* opaque, uint64_t prepared, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        PairingState& ps = pairing_state(b);
        require(ps.prepared.count(prepared) != 0, "unknown prepared G2 handle");
        DV_CUDA(cudaStreamSynchronize(b.stream));
        ps.prepared.erase(prepared);
    });
}

extern "C" int dvgpu_bn254_pairing_check_prepared(void* opaque, const uint8_t* g1, uint64_t prepared,
                                                  const uint32_t* q_index, const uint64_t* offsets, size_t equations,
                                                  uint8_t* verdicts, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        check_offsets(offsets, equations);
        const uint64_t terms = offsets[equations];
        require(verdicts && ((g1 && q_index) || !terms), "invalid pairing terms");
        PairingState& ps = pairing_state(b);
        const auto it = ps.prepared.find(prepared);
        require(it != ps.prepared.end(), "unknown prepared G2 handle");
        const PreparedG2& pg = *it->second;
        for (uint64_t t = 0; t < terms; ++t) require(q_index[t] < pg.n, "prepared G2 index out of range");
        const cudaStream_t st = b.stream;
        uint8_t* d_in = b.in_points.as<uint8_t>(64 * terms);
        DV_CUDA(cudaMemcpyAsync(d_in, g1, 64 * terms, cudaMemcpyHostToDevice, st));
        G1A* p = b.conv_points.as<G1A>(std::max<uint64_t>(1, terms));
        uint32_t* bad = b.err.as<uint32_t>(2);
        DV_CUDA(cudaMemsetAsync(bad, 0xff, 2 * sizeof(uint32_t), st));
        convert_points<Fq>(d_in, p, terms, bad, st);
        uint64_t* d_off = upload_offsets(b, offsets, equations, st);
        Fq2* mil = b.aux.as<Fq2>(6 * std::max<uint64_t>(1, std::max(terms, equations)));
        uint32_t* d_qidx = ps.qidx.as<uint32_t>(std::max<uint64_t>(1, terms));
        if (terms) DV_CUDA(cudaMemcpyAsync(d_qidx, q_index, 4 * terms, cudaMemcpyHostToDevice, st));
        const bool multi = miller_per_equation(terms);
        if (multi) {
            // with no terms every equation's value is one (the kernel reads only the offsets)
            k_miller_multi<<<group_blocks(equations), 128, 0, st>>>(p, d_qidx, pg.inf.view<uint32_t>(),
                                                                   pg.lines.view<Line>(), d_off, equations, mil);
            DV_LAUNCH();
        } else if (terms) {
            k_miller_multi<<<group_blocks(terms), 128, 0, st>>>(p, d_qidx, pg.inf.view<uint32_t>(),
                                                               pg.lines.view<Line>(), nullptr, terms, mil);
            DV_LAUNCH();
        }
        finish_equations(b, mil, multi ? nullptr : d_off, equations, verdicts, nullptr, bad, nullptr, st);
    });
}
