// Host-side BN254 arithmetic for the serial tail of each device operation:
// the window combination (Horner over c-bit windows) and normalisation to
// affine of an MSM result, a handful of points per call.  The bulk of every
// operation runs in the CUDA kernels; this is the counterpart of the
// reference's host-side projective_t::to_affine (native/src/icicle_msm.cu:417-421).
//
// Representation: 4 x 64-bit little-endian limbs in Montgomery form with
// R = 2^256 -- bit-identical to the device's 8 x 32-bit limbs, so device
// results are reinterpreted without conversion.
#pragma once
#include <cstdint>
#include <cstring>

namespace dvh {

typedef unsigned __int128 u128;

struct Fq {
    uint64_t v[4];
};

static const uint64_t QP[4] = {0x3c208c16d87cfd47ull, 0x97816a916871ca8dull, 0xb85045b68181585dull,
                               0x30644e72e131a029ull};
static const uint64_t QINV = 0x87d20782e4866389ull;  // -q^{-1} mod 2^64
static const uint64_t QONE[4] = {0xd35d438dc58f0d9dull, 0x0a78eb28f5c70b3dull, 0x666ea36f7879462cull,
                                 0x0e0a77c19a07df2full};
static const uint64_t QR2[4] = {0xf32cfc5b538afa89ull, 0xb5e71911d44501fbull, 0x47ab1eff0a417ff6ull,
                                0x06d89f71cab8351full};

inline bool q_geq(const uint64_t* a, const uint64_t* b) {
    for (int i = 3; i >= 0; --i) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return true;
}
inline void q_subp(uint64_t* a, const uint64_t* b) {
    uint64_t br = 0;
    for (int i = 0; i < 4; ++i) {
        u128 d = (u128)a[i] - b[i] - br;
        a[i] = (uint64_t)d;
        br = (uint64_t)(d >> 64) & 1;
    }
}
inline Fq mul(const Fq& a, const Fq& b) {
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
        const uint64_t m = t[0] * QINV;
        c = ((u128)m * QP[0] + t[0]) >> 64;
        for (int j = 1; j < 4; ++j) {
            c += (u128)m * QP[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    Fq r = {{t[0], t[1], t[2], t[3]}};
    if (t[4] || q_geq(r.v, QP)) q_subp(r.v, QP);
    return r;
}
inline Fq add(const Fq& a, const Fq& b) {
    Fq r;
    uint64_t c = 0;
    for (int i = 0; i < 4; ++i) {
        u128 s = (u128)a.v[i] + b.v[i] + c;
        r.v[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    if (c || q_geq(r.v, QP)) q_subp(r.v, QP);
    return r;
}
inline Fq sub(const Fq& a, const Fq& b) {
    Fq r = a;
    if (q_geq(a.v, b.v)) {
        q_subp(r.v, b.v);
        return r;
    }
    uint64_t c = 0;
    for (int i = 0; i < 4; ++i) {
        u128 s = (u128)r.v[i] + QP[i] + c;
        r.v[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    q_subp(r.v, b.v);
    return r;
}
inline bool is_zero(const Fq& a) { return !(a.v[0] | a.v[1] | a.v[2] | a.v[3]); }
inline bool eq(const Fq& a, const Fq& b) { return !memcmp(a.v, b.v, 32); }
inline Fq zero() { Fq z = {{0, 0, 0, 0}}; return z; }
inline Fq one() { Fq r; memcpy(r.v, QONE, 32); return r; }
inline Fq dbl(const Fq& a) { return add(a, a); }
inline Fq neg(const Fq& a) { return is_zero(a) ? a : sub(zero(), a); }
inline Fq inv(const Fq& a) {
    const uint64_t e[4] = {QP[0] - 2, QP[1], QP[2], QP[3]};
    Fq r = one();
    for (int i = 255; i >= 0; --i) {
        r = mul(r, r);
        if ((e[i / 64] >> (i % 64)) & 1) r = mul(r, a);
    }
    return r;
}
inline Fq from_canonical(const uint64_t* c) {
    Fq a, r2;
    memcpy(a.v, c, 32);
    memcpy(r2.v, QR2, 32);
    return mul(a, r2);
}
inline void to_canonical(const Fq& a, uint8_t* out) {
    Fq one_raw = {{1, 0, 0, 0}};
    Fq r = mul(a, one_raw);
    for (int i = 0; i < 4; ++i)
        for (int b = 0; b < 8; ++b) out[8 * i + b] = (uint8_t)(r.v[i] >> (8 * b));
}

struct Fq2 {
    Fq c0, c1;
};
inline Fq2 mul(const Fq2& a, const Fq2& b) {
    const Fq t0 = mul(a.c0, b.c0), t1 = mul(a.c1, b.c1);
    const Fq t2 = mul(add(a.c0, a.c1), add(b.c0, b.c1));
    return {sub(t0, t1), sub(sub(t2, t0), t1)};
}
inline Fq2 add(const Fq2& a, const Fq2& b) { return {add(a.c0, b.c0), add(a.c1, b.c1)}; }
inline Fq2 sub(const Fq2& a, const Fq2& b) { return {sub(a.c0, b.c0), sub(a.c1, b.c1)}; }
inline Fq2 dbl(const Fq2& a) { return {dbl(a.c0), dbl(a.c1)}; }
inline bool is_zero(const Fq2& a) { return is_zero(a.c0) && is_zero(a.c1); }
inline Fq2 inv(const Fq2& a) {
    const Fq n = add(mul(a.c0, a.c0), mul(a.c1, a.c1));
    const Fq ni = inv(n);
    return {mul(a.c0, ni), neg(mul(a.c1, ni))};
}
inline void to_canonical(const Fq2& a, uint8_t* out) {
    to_canonical(a.c0, out);
    to_canonical(a.c1, out + 32);
}

// XYZZ points, same layout as the device struct (x, y, zz, zzz).
template <class F>
struct XYZZ {
    F x, y, zz, zzz;
};

template <class F>
inline XYZZ<F> xyzz_inf() {
    XYZZ<F> r;
    memset(&r, 0, sizeof r);
    return r;
}

template <class F>
inline XYZZ<F> xyzz_dbl(const XYZZ<F>& p) {
    if (is_zero(p.zz)) return p;
    const F u = dbl(p.y), v = mul(u, u), w = mul(u, v), s = mul(p.x, v);
    const F x2 = mul(p.x, p.x), m = add(dbl(x2), x2);
    const F x3 = sub(mul(m, m), dbl(s));
    const F y3 = sub(mul(m, sub(s, x3)), mul(w, p.y));
    return {x3, y3, mul(v, p.zz), mul(w, p.zzz)};
}

template <class F>
inline XYZZ<F> xyzz_add(const XYZZ<F>& p, const XYZZ<F>& q) {
    if (is_zero(p.zz)) return q;
    if (is_zero(q.zz)) return p;
    const F u1 = mul(p.x, q.zz), u2 = mul(q.x, p.zz);
    const F s1 = mul(p.y, q.zzz), s2 = mul(q.y, p.zzz);
    const F pp_ = sub(u2, u1), r = sub(s2, s1);
    if (is_zero(pp_)) {
        if (is_zero(r)) return xyzz_dbl(p);
        return xyzz_inf<F>();
    }
    const F pp = mul(pp_, pp_), ppp = mul(pp_, pp), qq = mul(u1, pp);
    const F x3 = sub(sub(mul(r, r), ppp), dbl(qq));
    const F y3 = sub(mul(r, sub(qq, x3)), mul(s1, ppp));
    return {x3, y3, mul(mul(p.zz, q.zz), pp), mul(mul(p.zzz, q.zzz), ppp)};
}

// Canonical affine bytes (x || y), all-zero for infinity.
template <class F>
inline void xyzz_to_affine_bytes(const XYZZ<F>& p, uint8_t* out) {
    if (is_zero(p.zz)) {
        memset(out, 0, 2 * sizeof(F));
        return;
    }
    const F d = inv(mul(p.zz, p.zzz));
    const F x = mul(p.x, mul(d, p.zzz));
    const F y = mul(p.y, mul(d, p.zz));
    to_canonical(x, out);
    to_canonical(y, out + sizeof(F));
}

// Canonical affine bytes of n points with one inversion (Montgomery's
// simultaneous-inversion trick over the non-infinite points).
template <class F>
inline void xyzz_batch_to_affine_bytes(const XYZZ<F>* p, size_t n, uint8_t* out) {
    F* pre = new F[n + 1];
    pre[0] = one();
    for (size_t i = 0; i < n; ++i) pre[i + 1] = is_zero(p[i].zz) ? pre[i] : mul(pre[i], mul(p[i].zz, p[i].zzz));
    F acc = inv(pre[n]);  // 1 / prod (zz zzz)
    for (size_t i = n; i-- > 0;) {
        uint8_t* o = out + 2 * sizeof(F) * i;
        if (is_zero(p[i].zz)) {
            memset(o, 0, 2 * sizeof(F));
            continue;
        }
        const F d = mul(acc, pre[i]);  // 1 / (zz zzz) of point i
        acc = mul(acc, mul(p[i].zz, p[i].zzz));
        to_canonical(mul(p[i].x, mul(d, p[i].zzz)), o);
        to_canonical(mul(p[i].y, mul(d, p[i].zz)), o + sizeof(F));
    }
    delete[] pre;
}

}  // namespace dvh
