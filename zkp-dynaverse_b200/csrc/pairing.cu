// BN254 optimal ate pairing and pairing-product checks on sm_100a.
//
// The verifier's checks (crates/protocol/src/verification.rs:37-144):
// PairingChecks::equal / equal_prepared / product_equal reduce one equation
// to prod_k e(P_k, Q_k) = 1 (right-hand G1 points negated by the caller),
// computed by Bn254::multi_miller_loop and final_exponentiation.  Here a
// launch takes many equations: one thread per term runs the Miller loop,
// one thread per equation multiplies its terms' values and runs the final
// exponentiation.  The reference's native Miller probe
// (native/include/dynaverse_bn254_miller.h) is a diagnostic of line traces
// and is not reproduced.
//
// Tower: Fq2 = Fq[u]/(u^2 + 1), Fq6 = Fq2[v]/(v^3 - xi), Fq12 = Fq6[w]/(w^2 - v),
// xi = 9 + u; the coefficient of w^j (c0.c0 = w^0, c0.c1 = w^2, c0.c2 = w^4,
// c1.c0 = w^1, c1.c1 = w^3, c1.c2 = w^5) maps under the q-power Frobenius
// to conj(a) xi^(j(q-1)/6).
//
// Miller loop over the NAF of 6z + 2 (z the BN seed), then the lines to
// pi(Q) and -pi^2(Q).  T is kept in Jacobian coordinates on the twist
// E': y^2 = x^3 + 3/xi, untwisted by (x, y) -> (x w^2, y w^3).  The line
// through T (slope lam) at P = (xp, yp) is yp - lam xp w + (lam xT - yT) w^3;
// each step multiplies it by a nonzero Fq2 factor (killed by the final
// exponentiation, since Fq2* lies in the kernel of q^6 - 1):
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
// cyclotomic subgroup).  A verdict is result == 1; the value written for a
// single pairing is the GT element in the tower order above, canonical.
#include <cstring>
#include <string>
#include <vector>

#include "abi_util.hpp"
#include "backend.hpp"

namespace dv {
namespace {

// Out-of-line tower functions take their operands by const reference: a
// 384-byte Fq12 passed by value into a __noinline__ function that hands it
// on to further __noinline__ calls came back altered on sm_100a (nvcc 12.9);
// by reference it is never copied.
struct Fq6 {
    Fq2 c0, c1, c2;
};
struct Fq12 {
    Fq6 c0, c1;
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
constexpr uint64_t BN_Z = 4965661367192848881ull;

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

DV_INL Fq6 f6_add(const Fq6& a, const Fq6& b) { return {Fq2::add(a.c0, b.c0), Fq2::add(a.c1, b.c1), Fq2::add(a.c2, b.c2)}; }
DV_INL Fq6 f6_sub(const Fq6& a, const Fq6& b) { return {Fq2::sub(a.c0, b.c0), Fq2::sub(a.c1, b.c1), Fq2::sub(a.c2, b.c2)}; }
DV_INL Fq6 f6_neg(const Fq6& a) { return {Fq2::neg(a.c0), Fq2::neg(a.c1), Fq2::neg(a.c2)}; }
DV_INL Fq6 f6_mul_v(const Fq6& a) { return {mul_xi(a.c2), a.c0, a.c1}; }

// Karatsuba over v^3 = xi: 6 Fq2 products.
__device__ __noinline__ Fq6 f6_mul(const Fq6& a, const Fq6& b) {
    const Fq2 v0 = Fq2::mul(a.c0, b.c0), v1 = Fq2::mul(a.c1, b.c1), v2 = Fq2::mul(a.c2, b.c2);
    const Fq2 t0 = Fq2::mul(Fq2::add(a.c1, a.c2), Fq2::add(b.c1, b.c2));
    const Fq2 t1 = Fq2::mul(Fq2::add(a.c0, a.c1), Fq2::add(b.c0, b.c1));
    const Fq2 t2 = Fq2::mul(Fq2::add(a.c0, a.c2), Fq2::add(b.c0, b.c2));
    return {Fq2::add(v0, mul_xi(Fq2::sub(Fq2::sub(t0, v1), v2))),
            Fq2::add(Fq2::sub(Fq2::sub(t1, v0), v1), mul_xi(v2)),
            Fq2::add(Fq2::sub(Fq2::sub(t2, v0), v2), v1)};
}
// (x0 + x1 v + x2 v^2)(b0 + b1 v): 5 Fq2 products.
__device__ __noinline__ Fq6 f6_mul_01(const Fq6& x, const Fq2& b0, const Fq2& b1) {
    const Fq2 v0 = Fq2::mul(x.c0, b0), v1 = Fq2::mul(x.c1, b1);
    const Fq2 t = Fq2::mul(Fq2::add(x.c0, x.c1), Fq2::add(b0, b1));
    return {Fq2::add(v0, mul_xi(Fq2::mul(x.c2, b1))), Fq2::sub(Fq2::sub(t, v0), v1),
            Fq2::add(v1, Fq2::mul(x.c2, b0))};
}
__device__ __noinline__ Fq6 f6_inv(const Fq6& a) {
    const Fq2 t0 = Fq2::sub(Fq2::sqr(a.c0), mul_xi(Fq2::mul(a.c1, a.c2)));
    const Fq2 t1 = Fq2::sub(mul_xi(Fq2::sqr(a.c2)), Fq2::mul(a.c0, a.c1));
    const Fq2 t2 = Fq2::sub(Fq2::sqr(a.c1), Fq2::mul(a.c0, a.c2));
    const Fq2 d = Fq2::add(Fq2::mul(a.c0, t0), mul_xi(Fq2::add(Fq2::mul(a.c2, t1), Fq2::mul(a.c1, t2))));
    const Fq2 di = Fq2::inv(d);
    return {Fq2::mul(t0, di), Fq2::mul(t1, di), Fq2::mul(t2, di)};
}

DV_INL Fq12 f12_one() {
    Fq12 r;
    r.c0 = {Fq2::one(), Fq2::zero(), Fq2::zero()};
    r.c1 = {Fq2::zero(), Fq2::zero(), Fq2::zero()};
    return r;
}
DV_INL Fq12 f12_conj(const Fq12& a) { return {a.c0, f6_neg(a.c1)}; }
// Karatsuba: 3 Fq6 products.
__device__ __noinline__ Fq12 f12_mul(const Fq12& a, const Fq12& b) {
    const Fq6 t0 = f6_mul(a.c0, b.c0), t1 = f6_mul(a.c1, b.c1);
    const Fq6 t2 = f6_mul(f6_add(a.c0, a.c1), f6_add(b.c0, b.c1));
    return {f6_add(t0, f6_mul_v(t1)), f6_sub(f6_sub(t2, t0), t1)};
}
// (g + h w)^2 = (g + h)(g + h v) - t - t v + 2 t w, t = g h: 2 Fq6 products.
__device__ __noinline__ Fq12 f12_sqr(const Fq12& a) {
    const Fq6 t = f6_mul(a.c0, a.c1);
    const Fq6 m = f6_mul(f6_add(a.c0, a.c1), f6_add(a.c0, f6_mul_v(a.c1)));
    return {f6_sub(f6_sub(m, t), f6_mul_v(t)), f6_add(t, t)};
}
// f (l0 + (l1 + l3 v) w) with l0 in Fq2 (the line's w^0 term), l1, l3 its
// w^1 and w^3 terms: 13 Fq2 products.
__device__ __noinline__ Fq12 f12_mul_line(const Fq12& f, const Fq2& l0, const Fq2& l1, const Fq2& l3) {
    const Fq6 t0 = {Fq2::mul(f.c0.c0, l0), Fq2::mul(f.c0.c1, l0), Fq2::mul(f.c0.c2, l0)};
    const Fq6 t1 = f6_mul_01(f.c1, l1, l3);
    const Fq6 t2 = f6_mul_01(f6_add(f.c0, f.c1), Fq2::add(l0, l1), l3);
    return {f6_add(t0, f6_mul_v(t1)), f6_sub(f6_sub(t2, t0), t1)};
}
__device__ __noinline__ Fq12 f12_inv(const Fq12& a) {
    const Fq6 d = f6_inv(f6_sub(f6_mul(a.c0, a.c0), f6_mul_v(f6_mul(a.c1, a.c1))));
    return {f6_mul(a.c0, d), f6_neg(f6_mul(a.c1, d))};
}
// q^k-power Frobenius, k = 1, 2, 3.
__device__ __noinline__ Fq12 f12_frob(const Fq12& in, int k) {
    Fq12 a = in;
    Fq2* c = &a.c0.c0;
    const int wpow[6] = {0, 2, 4, 1, 3, 5};
    for (int i = 0; i < 6; ++i) {
        const int j = wpow[i];
        if (k == 2) {
            c[i] = Fq2::mul_fq(c[i], frob2(j));
        } else {
            Fq2 g = frob1(j);
            if (k == 3) g = Fq2::mul_fq(g, frob2(j));
            c[i] = Fq2::mul(Fq2::conj(c[i]), g);
        }
    }
    return a;
}
DV_INL bool f12_is_one(const Fq12& a) {
    const Fq2* c = &a.c0.c0;
    if (!(c[0].c0 == Fq::one()) || !c[0].c1.is_zero()) return false;
    for (int i = 1; i < 6; ++i)
        if (!c[i].is_zero()) return false;
    return true;
}
// a^z, z the BN seed (63 bits), left to right.
__device__ __noinline__ Fq12 f12_pow_z(const Fq12& a) {
    Fq12 r = a;
    for (int i = 61; i >= 0; --i) {
        r = f12_sqr(r);
        if ((BN_Z >> i) & 1) r = f12_mul(r, a);
    }
    return r;
}

struct Tw {
    Fq2 x, y, z;  // Jacobian on the twist
};

// T <- 2T; returns the line's (w^0, w^1, w^3) terms at P.
__device__ __noinline__ void dbl_step(Tw& t, const Fq& xp, const Fq& yp, Fq2& l0, Fq2& l1, Fq2& l3) {
    const Fq2 a = Fq2::sqr(t.x), b = Fq2::sqr(t.y), c = Fq2::sqr(b), zz = Fq2::sqr(t.z);
    const Fq2 e = Fq2::add(Fq2::dbl(a), a);
    const Fq2 d = Fq2::dbl(Fq2::sub(Fq2::sub(Fq2::sqr(Fq2::add(t.x, b)), a), c));
    const Fq2 z3 = Fq2::dbl(Fq2::mul(t.y, t.z));
    l0 = Fq2::mul_fq(Fq2::mul(z3, zz), yp);
    l1 = Fq2::neg(Fq2::mul_fq(Fq2::mul(e, zz), xp));
    l3 = Fq2::sub(Fq2::mul(e, t.x), Fq2::dbl(b));
    const Fq2 x3 = Fq2::sub(Fq2::sqr(e), Fq2::dbl(d));
    const Fq2 c8 = Fq2::dbl(Fq2::dbl(Fq2::dbl(c)));
    t.y = Fq2::sub(Fq2::mul(e, Fq2::sub(d, x3)), c8);
    t.x = x3;
    t.z = z3;
}
// T <- T + S (S affine); returns the line's terms at P.
__device__ __noinline__ void add_step(Tw& t, const Fq2& xs, const Fq2& ys, const Fq& xp, const Fq& yp, Fq2& l0,
                                      Fq2& l1, Fq2& l3) {
    const Fq2 zz = Fq2::sqr(t.z);
    const Fq2 h = Fq2::sub(Fq2::mul(xs, zz), t.x);
    const Fq2 r = Fq2::dbl(Fq2::sub(Fq2::mul(ys, Fq2::mul(t.z, zz)), t.y));
    const Fq2 hh = Fq2::sqr(h);
    const Fq2 i = Fq2::dbl(Fq2::dbl(hh));
    const Fq2 j = Fq2::mul(h, i);
    const Fq2 v = Fq2::mul(t.x, i);
    const Fq2 z3 = Fq2::sub(Fq2::sub(Fq2::sqr(Fq2::add(t.z, h)), zz), hh);
    l0 = Fq2::mul_fq(z3, yp);
    l1 = Fq2::neg(Fq2::mul_fq(r, xp));
    l3 = Fq2::sub(Fq2::mul(r, xs), Fq2::mul(z3, ys));
    const Fq2 x3 = Fq2::sub(Fq2::sub(Fq2::sqr(r), j), Fq2::dbl(v));
    t.y = Fq2::sub(Fq2::mul(r, Fq2::sub(v, x3)), Fq2::dbl(Fq2::mul(t.y, j)));
    t.x = x3;
    t.z = z3;
}

__device__ Fq12 miller_loop(const G1A& p, const G2A& q) {
    Tw t{q.x, q.y, Fq2::one()};
    Fq12 f = f12_one();
    Fq2 l0, l1, l3;
    const Fq2 nqy = Fq2::neg(q.y);
    for (int i = 1; i < NAF_LEN; ++i) {
        dbl_step(t, p.x, p.y, l0, l1, l3);
        f = f12_mul_line(f12_sqr(f), l0, l1, l3);
        const int d = NAF_6Z2[i];
        if (d) {
            add_step(t, q.x, d > 0 ? q.y : nqy, p.x, p.y, l0, l1, l3);
            f = f12_mul_line(f, l0, l1, l3);
        }
    }
    // pi(Q) = (conj(x) xi^((q-1)/3), conj(y) xi^((q-1)/2)); -pi^2(Q) = (x xi^((q^2-1)/3), -y xi^((q^2-1)/2))
    const Fq2 x1 = Fq2::mul(Fq2::conj(q.x), frob1(2)), y1 = Fq2::mul(Fq2::conj(q.y), frob1(3));
    const Fq2 x2 = Fq2::mul_fq(q.x, frob2(2)), y2 = Fq2::neg(Fq2::mul_fq(q.y, frob2(3)));
    add_step(t, x1, y1, p.x, p.y, l0, l1, l3);
    f = f12_mul_line(f, l0, l1, l3);
    add_step(t, x2, y2, p.x, p.y, l0, l1, l3);
    return f12_mul_line(f, l0, l1, l3);
}

__device__ Fq12 final_exponentiation(const Fq12& m) {
    Fq12 f = f12_mul(f12_conj(m), f12_inv(m));  // ^(q^6 - 1)
    f = f12_mul(f12_frob(f, 2), f);             // ^(q^2 + 1)
    const Fq12 a = f12_pow_z(f);
    const Fq12 b = f12_pow_z(a);
    const Fq12 c = f12_pow_z(b);
    const Fq12 a2 = f12_sqr(a), a4 = f12_sqr(a2), a6 = f12_mul(a4, a2);
    const Fq12 b2 = f12_sqr(b), b6 = f12_mul(f12_sqr(b2), b2), b12 = f12_sqr(b6);
    const Fq12 c4 = f12_sqr(f12_sqr(c)), c12 = f12_mul(f12_sqr(c4), c4);
    const Fq12 tt = f12_mul(c12, b6);
    const Fq12 l1 = f12_mul(tt, a4);
    const Fq12 l2 = f12_mul(tt, a6);
    const Fq12 l3 = f12_mul(l1, f12_conj(f));
    const Fq12 l0 = f12_mul(f12_mul(f12_mul(c12, b12), a6), f);
    Fq12 r = f12_mul(l0, f12_frob(l1, 1));
    r = f12_mul(r, f12_frob(l2, 2));
    return f12_mul(r, f12_frob(l3, 3));
}

// Miller value of every term (one thread each); infinity on either side gives one.
__global__ void __launch_bounds__(128) k_miller(const G1A* __restrict__ g1, const G2A* __restrict__ g2,
                                                uint64_t terms, Fq12* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= terms) return;
    const G1A p = g1[i];
    const G2A q = g2[i];
    out[i] = (p.is_inf() || q.is_inf()) ? f12_one() : miller_loop(p, q);
}

// Per equation: product of its terms' values, final exponentiation; the
// verdict (result == 1) and, with gt, the canonical GT element.
__global__ void __launch_bounds__(128) k_final_exp(const Fq12* __restrict__ miller, const uint64_t* __restrict__ offsets,
                                                   uint64_t equations, uint8_t* __restrict__ verdicts,
                                                   uint8_t* __restrict__ gt) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= equations) return;
    Fq12 f = f12_one();
    for (uint64_t k = offsets[e]; k < offsets[e + 1]; ++k) f = f12_mul(f, miller[k]);
    const Fq12 r = final_exponentiation(f);
    if (verdicts) verdicts[e] = f12_is_one(r) ? 1 : 0;
    if (gt) {
        const Fq2* c = &r.c0.c0;
        for (int i = 0; i < 6; ++i) {
            store_canonical(gt + 384 * e + 64 * i, c[i].c0);
            store_canonical(gt + 384 * e + 64 * i + 32, c[i].c1);
        }
    }
}

void pairing_run(Backend& b, const uint8_t* g1, const uint8_t* g2, uint64_t terms, const uint64_t* offsets,
                 uint64_t equations, uint8_t* verdicts, uint8_t* gt, cudaStream_t st) {
    uint8_t* d_in = b.in_points.as<uint8_t>(192 * terms);
    DV_CUDA(cudaMemcpyAsync(d_in, g1, 64 * terms, cudaMemcpyHostToDevice, st));
    DV_CUDA(cudaMemcpyAsync(d_in + 64 * terms, g2, 128 * terms, cudaMemcpyHostToDevice, st));
    G1A* p = b.conv_points.as<G1A>(terms * 3);  // G1A (64 B) then G2A (128 B)
    G2A* q = reinterpret_cast<G2A*>(p + terms);
    uint32_t* bad = b.err.as<uint32_t>(2);
    DV_CUDA(cudaMemsetAsync(bad, 0xff, 2 * sizeof(uint32_t), st));
    convert_points<Fq>(d_in, p, terms, bad, st);
    convert_points<Fq2>(d_in + 64 * terms, q, terms, bad + 1, st);
    Fq12* mil = b.aux.as<Fq12>(terms);
    if (terms) {
        k_miller<<<(unsigned)((terms + 127) / 128), 128, 0, st>>>(p, q, terms, mil);
        DV_LAUNCH();
    }
    uint64_t* d_off = b.idx.as<uint64_t>(equations + 1);
    DV_CUDA(cudaMemcpyAsync(d_off, offsets, 8 * (equations + 1), cudaMemcpyHostToDevice, st));
    // GT elements first (16-byte aligned stores), then the verdict bytes
    uint8_t* d_gt = b.out_buf.as<uint8_t>(equations * ((gt ? 384 : 0) + 1));
    uint8_t* d_out = d_gt + (gt ? 384 * equations : 0);
    k_final_exp<<<(unsigned)((equations + 127) / 128), 128, 0, st>>>(mil, d_off, equations, d_out,
                                                                     gt ? d_gt : nullptr);
    DV_LAUNCH();
    uint32_t hbad[2];
    DV_CUDA(cudaMemcpyAsync(hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st));
    DV_CUDA(cudaStreamSynchronize(st));
    if (hbad[0] != 0xffffffffu) throw InvalidArgument("invalid G1 point at term " + std::to_string(hbad[0]));
    if (hbad[1] != 0xffffffffu) throw InvalidArgument("invalid G2 point at term " + std::to_string(hbad[1]));
    if (verdicts) DV_CUDA(cudaMemcpy(verdicts, d_out, equations, cudaMemcpyDeviceToHost));
    if (gt) DV_CUDA(cudaMemcpy(gt, d_gt, 384 * equations, cudaMemcpyDeviceToHost));
}

}  // namespace
}  // namespace dv

using namespace dv;

extern "C" int dvgpu_bn254_pairing_check(void* opaque, const uint8_t* g1, const uint8_t* g2, const uint64_t* offsets,
                                         size_t equations, uint8_t* verdicts, char* error, size_t cap) {
    return guarded(opaque, error, cap, [&](Backend& b) {
        require(offsets && verdicts && equations >= 1 && equations <= (1u << 24), "invalid pairing check arguments");
        require(offsets[0] == 0, "pairing offsets must start at 0");
        for (size_t e = 0; e < equations; ++e) require(offsets[e + 1] >= offsets[e], "pairing offsets must not decrease");
        const uint64_t terms = offsets[equations];
        require(terms <= (1u << 24) && (g1 || !terms) && (g2 || !terms), "invalid pairing terms");
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
