// BN254 G1 (y^2 = x^3 + 3 over Fq) and G2 (twist y^2 = x^3 + 3/(9+u) over
// Fq2) in XYZZ coordinates: x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2, ZZ = 0 is the
// point at infinity.  Formulas are the a = 0 specialisations of the
// Explicit-Formulas Database "xyzz" family (madd-2008-s, add-2008-s,
// dbl-2008-s-1, mdbl-2008-s-1): mixed add 8M+2S, full add 12M+2S,
// double 6M+3S.  Affine infinity is encoded as (0, 0), which is on neither
// curve.
#pragma once
#include "field.cuh"

namespace dv {

template <class F>
struct Affine {
    F x, y;
    DV_INL bool is_inf() const { return x.is_zero() && y.is_zero(); }
    DV_INL static Affine inf() { return {F::zero(), F::zero()}; }
    DV_INL Affine neg() const { return {x, F::neg(y)}; }
};

template <class F>
struct XYZZ {
    F x, y, zz, zzz;

    DV_INL static XYZZ inf() { return {F::one(), F::one(), F::zero(), F::zero()}; }
    DV_INL bool is_inf() const { return zz.is_zero(); }
    DV_INL static XYZZ from_affine(const Affine<F>& a) {
        if (a.is_inf()) return inf();
        return {a.x, a.y, F::one(), F::one()};
    }
    DV_INL XYZZ neg() const { return {x, F::neg(y), zz, zzz}; }

    // 2 * (x, y) for an affine point (mdbl-2008-s-1).
    DV_INL static XYZZ dbl_affine(const Affine<F>& a) {
        const F u = F::dbl(a.y);
        const F v = F::sqr(u);
        const F w = F::mul(u, v);
        const F s = F::mul(a.x, v);
        const F x2 = F::sqr(a.x);
        const F m = F::add(F::dbl(x2), x2);
        const F x3 = F::sub(F::sqr(m), F::dbl(s));
        const F y3 = F::sub(F::mul(m, F::sub(s, x3)), F::mul(w, a.y));
        return {x3, y3, v, w};
    }

    // dbl-2008-s-1 (a = 0)
    DV_INL static XYZZ dbl(const XYZZ& p) {
        if (p.is_inf()) return p;
        const F u = F::dbl(p.y);
        const F v = F::sqr(u);
        const F w = F::mul(u, v);
        const F s = F::mul(p.x, v);
        const F x2 = F::sqr(p.x);
        const F m = F::add(F::dbl(x2), x2);
        const F x3 = F::sub(F::sqr(m), F::dbl(s));
        const F y3 = F::sub(F::mul(m, F::sub(s, x3)), F::mul(w, p.y));
        return {x3, y3, F::mul(v, p.zz), F::mul(w, p.zzz)};
    }

    // Rare case of add_affine: same x coordinate (doubling or P + (-P)), kept
    // out of line so the hot accumulation loop stays small.
    __device__ __noinline__ static XYZZ add_affine_equal_x(Affine<F> a, F r) {
        if (r.is_zero()) return dbl_affine(a);
        return inf();
    }

    // p + a with a affine (madd-2008-s).  Over Fq the ten products are
    // issued as five independent pairs (F::mul2): measured 7 % faster bucket
    // accumulation; over Fq2, whose products already hold three independent
    // chains, the plain sequence is faster.
    DV_INL static XYZZ add_affine(const XYZZ& p, const Affine<F>& a) {
        if (a.is_inf()) return p;
        if (p.is_inf()) return from_affine(a);
        if constexpr (sizeof(F) == sizeof(Fq)) {
            const auto us = F::mul2(a.x, p.zz, a.y, p.zzz);  // U2, S2
            const F pp_ = F::sub(us.r0, p.x);
            const F r = F::sub(us.r1, p.y);
            if (pp_.is_zero()) return add_affine_equal_x(a, r);
            const auto sq = F::sqr2(pp_, r);                   // PP, R^2
            const F pp = sq.r0;
            const auto pq = F::mul2(pp_, pp, p.x, pp);          // PPP, Q
            const F ppp = pq.r0, q = pq.r1;
            const F x3 = F::sub(F::sub(sq.r1, ppp), F::dbl(q));
            const auto zs = F::mul2(p.zz, pp, p.zzz, ppp);      // ZZ3, ZZZ3
            const auto ys = F::mul2(r, F::sub(q, x3), p.y, ppp);
            return {x3, F::sub(ys.r0, ys.r1), zs.r0, zs.r1};
        } else {
            const F u2 = F::mul(a.x, p.zz);
            const F s2 = F::mul(a.y, p.zzz);
            const F pp_ = F::sub(u2, p.x);
            const F r = F::sub(s2, p.y);
            if (pp_.is_zero()) return add_affine_equal_x(a, r);
            const F pp = F::sqr(pp_);
            const F ppp = F::mul(pp_, pp);
            const F q = F::mul(p.x, pp);
            const F x3 = F::sub(F::sub(F::sqr(r), ppp), F::dbl(q));
            const F y3 = F::sub(F::mul(r, F::sub(q, x3)), F::mul(p.y, ppp));
            return {x3, y3, F::mul(p.zz, pp), F::mul(p.zzz, ppp)};
        }
    }

    // p + q (add-2008-s).
    DV_INL static XYZZ add(const XYZZ& p, const XYZZ& q) {
        if (p.is_inf()) return q;
        if (q.is_inf()) return p;
        const F u1 = F::mul(p.x, q.zz);
        const F u2 = F::mul(q.x, p.zz);
        const F s1 = F::mul(p.y, q.zzz);
        const F s2 = F::mul(q.y, p.zzz);
        const F pp_ = F::sub(u2, u1);
        const F r = F::sub(s2, s1);
        if (pp_.is_zero()) {
            if (r.is_zero()) return dbl(p);
            return inf();
        }
        const F pp = F::sqr(pp_);
        const F ppp = F::mul(pp_, pp);
        const F qq = F::mul(u1, pp);
        const F x3 = F::sub(F::sub(F::sqr(r), ppp), F::dbl(qq));
        const F y3 = F::sub(F::mul(r, F::sub(qq, x3)), F::mul(s1, ppp));
        return {x3, y3, F::mul(F::mul(p.zz, q.zz), pp), F::mul(F::mul(p.zzz, q.zzz), ppp)};
    }

    // Over Fq: doubling and full addition with their products issued as
    // independent pairs (F::mul2), for the long dependent chains of a scalar
    // multiplication run by few threads (the G1 transform's butterflies).
    DV_INL static XYZZ dbl_paired(const XYZZ& p) {
        if (p.is_inf()) return p;
        const F u = F::dbl(p.y);
        const auto vx = F::sqr2(u, p.x);              // V = U^2, X^2
        const F v = vx.r0;
        const auto ws = F::mul2(u, v, p.x, v);         // W = U V, S = X V
        const F w = ws.r0, s = ws.r1;
        const F m = F::add(F::dbl(vx.r1), vx.r1);
        const auto mz = F::mul2(m, m, v, p.zz);        // M^2, ZZ3
        const F x3 = F::sub(mz.r0, F::dbl(s));
        const auto wy = F::mul2(w, p.y, w, p.zzz);     // W Y, ZZZ3
        const F y3 = F::sub(F::mul(m, F::sub(s, x3)), wy.r0);
        return {x3, y3, mz.r1, wy.r1};
    }
    DV_INL static XYZZ add_paired(const XYZZ& p, const XYZZ& q) {
        if (p.is_inf()) return q;
        if (q.is_inf()) return p;
        const auto u = F::mul2(p.x, q.zz, q.x, p.zz);  // U1, U2
        const auto s = F::mul2(p.y, q.zzz, q.y, p.zzz);  // S1, S2
        const F pp_ = F::sub(u.r1, u.r0);
        const F r = F::sub(s.r1, s.r0);
        if (pp_.is_zero()) {
            if (r.is_zero()) return dbl_paired(p);
            return inf();
        }
        const auto sq = F::sqr2(pp_, r);                // PP, R^2
        const F pp = sq.r0;
        const auto pq = F::mul2(pp_, pp, u.r0, pp);     // PPP, Q
        const F ppp = pq.r0, qq = pq.r1;
        const F x3 = F::sub(F::sub(sq.r1, ppp), F::dbl(qq));
        const auto zz = F::mul2(p.zz, q.zz, p.zzz, q.zzz);
        const auto zs = F::mul2(zz.r0, pp, zz.r1, ppp);  // ZZ3, ZZZ3
        const auto ys = F::mul2(r, F::sub(qq, x3), s.r0, ppp);
        return {x3, F::sub(ys.r0, ys.r1), zs.r0, zs.r1};
    }

    // Projective equality without normalisation.
    DV_INL static bool equal(const XYZZ& p, const XYZZ& q) {
        const bool pi = p.is_inf(), qi = q.is_inf();
        if (pi || qi) return pi && qi;
        return F::mul(p.x, q.zz) == F::mul(q.x, p.zz) && F::mul(p.y, q.zzz) == F::mul(q.y, p.zzz);
    }

    DV_INL Affine<F> to_affine() const {
        if (is_inf()) return Affine<F>::inf();
        const F d = F::inv(F::mul(zz, zzz));     // 1 / (ZZ * ZZZ)
        const F izz = F::mul(d, zzz);            // 1 / ZZ
        const F izzz = F::mul(d, zz);            // 1 / ZZZ
        return {F::mul(x, izz), F::mul(y, izzz)};
    }
};

// ------------------------------------------------------------- warp helpers
DV_INL Fq shfl_up(const Fq& a, int d) {
    Fq r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_up_sync(0xffffffffu, a.v[i], d);
    return r;
}
DV_INL Fq shfl_down(const Fq& a, int d) {
    Fq r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_down_sync(0xffffffffu, a.v[i], d);
    return r;
}
DV_INL Fq shfl_idx(const Fq& a, int l) {
    Fq r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_sync(0xffffffffu, a.v[i], l);
    return r;
}
DV_INL Fq2 shfl_up(const Fq2& a, int d) { return {shfl_up(a.c0, d), shfl_up(a.c1, d)}; }
DV_INL Fq2 shfl_down(const Fq2& a, int d) { return {shfl_down(a.c0, d), shfl_down(a.c1, d)}; }
DV_INL Fq2 shfl_idx(const Fq2& a, int l) { return {shfl_idx(a.c0, l), shfl_idx(a.c1, l)}; }

// Warp-wide simultaneous inversion: returns 1/x for every lane (x != 0).
template <class F>
DV_INL F warp_batch_inverse(const F& x) {
    const int lane = threadIdx.x & 31;
    F pre = x;  // inclusive prefix product
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const F o = shfl_up(pre, d);
        if (lane >= d) pre = F::mul(pre, o);
    }
    F suf = x;  // inclusive suffix product
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const F o = shfl_down(suf, d);
        if (lane + d < 32) suf = F::mul(suf, o);
    }
    F total_inv = F::inv(shfl_idx(pre, 31));
    F excl_pre = shfl_up(pre, 1);
    F excl_suf = shfl_down(suf, 1);
    if (lane == 0) excl_pre = F::one();
    if (lane == 31) excl_suf = F::one();
    return F::mul(total_inv, F::mul(excl_pre, excl_suf));
}

typedef Affine<Fq> G1A;
typedef XYZZ<Fq> G1X;
typedef Affine<Fq2> G2A;
typedef XYZZ<Fq2> G2X;

// ------------------------------------------------------------- canonical I/O
// Canonical little-endian 32-byte field elements, read as 8 u32 words.

DV_INL void load_words(const uint8_t* p, uint32_t* w) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    const uint4 a = q[0], b = q[1];
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}
DV_INL void store_words(uint8_t* p, const uint32_t* w) {
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(w[0], w[1], w[2], w[3]);
    q[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// Montgomery field element -> canonical little-endian bytes (Fq2: c0, c1).
DV_INL void store_canonical(uint8_t* out, const Fq& a) {
    uint32_t c[8];
    a.to_canonical(c);
    store_words(out, c);
}
DV_INL void store_canonical(uint8_t* out, const Fq2& a) {
    store_canonical(out, a.c0);
    store_canonical(out + 32, a.c1);
}

// Curve equations (Montgomery constants).
DV_INL Fq g1_b() {
    uint32_t c[8] = {3, 0, 0, 0, 0, 0, 0, 0};
    return Fq::from_canonical(c);
}
DV_INL Fq2 g2_b() {
    // 3 / (9 + u), canonical limbs.
    const uint32_t c0[8] = {0x24a138e5u, 0x3267e6dcu, 0x59dbefa3u, 0xb5b4c5e5u,
                            0x1be06ac3u, 0x81be1899u, 0xceb8aaaeu, 0x2b149d40u};
    const uint32_t c1[8] = {0x85c315d2u, 0xe4a2bd06u, 0xe52d1852u, 0xa74fa084u,
                            0xeed8fdf4u, 0xcd2cafadu, 0x3af0fed4u, 0x009713b0u};
    return {Fq::from_canonical(c0), Fq::from_canonical(c1)};
}

template <class F>
struct CurveOps;
template <>
struct CurveOps<Fq> {
    DV_INL static bool on_curve(const Affine<Fq>& a) {
        if (a.is_inf()) return true;
        return Fq::sqr(a.y) == Fq::add(Fq::mul(Fq::sqr(a.x), a.x), g1_b());
    }
};
template <>
struct CurveOps<Fq2> {
    DV_INL static bool on_curve(const Affine<Fq2>& a) {
        if (a.is_inf()) return true;
        return Fq2::sqr(a.y) == Fq2::add(Fq2::mul(Fq2::sqr(a.x), a.x), g2_b());
    }
};

}  // namespace dv
