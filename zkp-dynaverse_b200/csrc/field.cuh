// BN254 prime fields on sm_100a: 8 x 32-bit limbs, Montgomery form R = 2^256.
//
// Multiplication is CIOS (Koc, Acar, Kaliski, "Analyzing and comparing
// Montgomery multiplication algorithms", 1996) written as PTX carry chains.
// Each row "t += x * v" is split into an even-limb chain (lo of v0,v2,.. into
// t0,t2,..; hi into t1,t3,..) and an odd-limb chain, so every chain is a
// single uninterrupted mad.lo.cc / madc.hi.cc sequence.  p < 2^254, so the
// 9-limb accumulator never overflows (T < 2p before each row, and
// T + a*b_i + m*p < 2^288).
//
// Values are kept fully reduced in [0, p).
#pragma once
#include <cstdint>

namespace dv {

struct FqCfg {
    static constexpr uint32_t P0 = 0xd87cfd47u, P1 = 0x3c208c16u, P2 = 0x6871ca8du, P3 = 0x97816a91u,
                              P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
    static constexpr uint32_t INV = 0xe4866389u;  // -p^{-1} mod 2^32
    static constexpr uint32_t ONE0 = 0xc58f0d9du, ONE1 = 0xd35d438du, ONE2 = 0xf5c70b3du, ONE3 = 0x0a78eb28u, ONE4 = 0x7879462cu, ONE5 = 0x666ea36fu, ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
    static constexpr uint32_t R20 = 0x538afa89u, R21 = 0xf32cfc5bu, R22 = 0xd44501fbu, R23 = 0xb5e71911u, R24 = 0x0a417ff6u, R25 = 0x47ab1effu, R26 = 0xcab8351fu, R27 = 0x06d89f71u;
    static constexpr uint32_t R30 = 0xda1530dfu, R31 = 0xb1cd6dafu, R32 = 0xa7283db6u, R33 = 0x62f210e6u, R34 = 0x0ada0afbu, R35 = 0xef7f0b0cu, R36 = 0x2d592544u, R37 = 0x20fd6e90u;
};
struct FrCfg {
    static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u,
                              P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
    static constexpr uint32_t INV = 0xefffffffu;
    static constexpr uint32_t ONE0 = 0x4ffffffbu, ONE1 = 0xac96341cu, ONE2 = 0x9f60cd29u, ONE3 = 0x36fc7695u, ONE4 = 0x7879462eu, ONE5 = 0x666ea36fu, ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
    static constexpr uint32_t R20 = 0xae216da7u, R21 = 0x1bb8e645u, R22 = 0xe35c59e3u, R23 = 0x53fe3ab1u, R24 = 0x53bb8085u, R25 = 0x8c49833du, R26 = 0x7f4e44a5u, R27 = 0x0216d0b1u;
    static constexpr uint32_t R30 = 0xb4bf0040u, R31 = 0x5e94d8e1u, R32 = 0x1cfbb6b8u, R33 = 0x2a489cbeu, R34 = 0xa19fcfedu, R35 = 0x893cc664u, R36 = 0x7fcc657cu, R37 = 0x0cf8594bu;
};

#define DV_INL __device__ __forceinline__

// Two results of a paired multiplication.
template <class T>
struct PairOf {
    T r0, r1;
};

template <class C>
struct __align__(16) Fp {  // 16-byte aligned: global copies move as 128-bit accesses
    uint32_t v[8];

    DV_INL static Fp zero() {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; ++i) r.v[i] = 0;
        return r;
    }
    DV_INL static Fp one() {
        Fp r;
        r.v[0] = C::ONE0; r.v[1] = C::ONE1; r.v[2] = C::ONE2; r.v[3] = C::ONE3;
        r.v[4] = C::ONE4; r.v[5] = C::ONE5; r.v[6] = C::ONE6; r.v[7] = C::ONE7;
        return r;
    }
    // R^2 mod p: the Montgomery form of R.
    DV_INL static Fp r2() {
        Fp r;
        r.v[0] = C::R20; r.v[1] = C::R21; r.v[2] = C::R22; r.v[3] = C::R23;
        r.v[4] = C::R24; r.v[5] = C::R25; r.v[6] = C::R26; r.v[7] = C::R27;
        return r;
    }
    DV_INL bool is_zero() const {
        uint32_t x = v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7];
        return x == 0;
    }
    DV_INL bool operator==(const Fp& o) const {
        uint32_t x = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) x |= v[i] ^ o.v[i];
        return x == 0;
    }

    // r = a - p if a >= p else a   (a < 2^256)
    DV_INL static void reduce_once(uint32_t* t) {
        uint32_t s[8], borrow;
        asm("sub.cc.u32 %0, %9, %17;\n\t"
            "subc.cc.u32 %1, %10, %18;\n\t"
            "subc.cc.u32 %2, %11, %19;\n\t"
            "subc.cc.u32 %3, %12, %20;\n\t"
            "subc.cc.u32 %4, %13, %21;\n\t"
            "subc.cc.u32 %5, %14, %22;\n\t"
            "subc.cc.u32 %6, %15, %23;\n\t"
            "subc.cc.u32 %7, %16, %24;\n\t"
            "subc.u32 %8, 0, 0;"
            : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]),
              "=r"(s[7]), "=r"(borrow)
            : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
              "n"(C::P0), "n"(C::P1), "n"(C::P2), "n"(C::P3), "n"(C::P4), "n"(C::P5), "n"(C::P6),
              "n"(C::P7));
        // borrow == 0xffffffff  <=>  t < p  -> keep t
#pragma unroll
        for (int i = 0; i < 8; ++i) t[i] = borrow ? t[i] : s[i];
    }

    DV_INL static Fp add(const Fp& a, const Fp& b) {
        Fp r;
        asm("add.cc.u32 %0, %8, %16;\n\t"
            "addc.cc.u32 %1, %9, %17;\n\t"
            "addc.cc.u32 %2, %10, %18;\n\t"
            "addc.cc.u32 %3, %11, %19;\n\t"
            "addc.cc.u32 %4, %12, %20;\n\t"
            "addc.cc.u32 %5, %13, %21;\n\t"
            "addc.cc.u32 %6, %14, %22;\n\t"
            "addc.u32 %7, %15, %23;"
            : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
              "=r"(r.v[6]), "=r"(r.v[7])
            : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
              "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
              "r"(b.v[6]), "r"(b.v[7]));
        reduce_once(r.v);
        return r;
    }

    DV_INL static Fp sub(const Fp& a, const Fp& b) {
        Fp r;
        uint32_t borrow;
        asm("sub.cc.u32 %0, %9, %17;\n\t"
            "subc.cc.u32 %1, %10, %18;\n\t"
            "subc.cc.u32 %2, %11, %19;\n\t"
            "subc.cc.u32 %3, %12, %20;\n\t"
            "subc.cc.u32 %4, %13, %21;\n\t"
            "subc.cc.u32 %5, %14, %22;\n\t"
            "subc.cc.u32 %6, %15, %23;\n\t"
            "subc.cc.u32 %7, %16, %24;\n\t"
            "subc.u32 %8, 0, 0;"
            : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
              "=r"(r.v[6]), "=r"(r.v[7]), "=r"(borrow)
            : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
              "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
              "r"(b.v[6]), "r"(b.v[7]));
        // add back p & borrow
        asm("add.cc.u32 %0, %0, %8;\n\t"
            "addc.cc.u32 %1, %1, %9;\n\t"
            "addc.cc.u32 %2, %2, %10;\n\t"
            "addc.cc.u32 %3, %3, %11;\n\t"
            "addc.cc.u32 %4, %4, %12;\n\t"
            "addc.cc.u32 %5, %5, %13;\n\t"
            "addc.cc.u32 %6, %6, %14;\n\t"
            "addc.u32 %7, %7, %15;"
            : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]),
              "+r"(r.v[6]), "+r"(r.v[7])
            : "r"(C::P0 & borrow), "r"(C::P1 & borrow), "r"(C::P2 & borrow), "r"(C::P3 & borrow),
              "r"(C::P4 & borrow), "r"(C::P5 & borrow), "r"(C::P6 & borrow), "r"(C::P7 & borrow));
        return r;
    }

    DV_INL static Fp dbl(const Fp& a) { return add(a, a); }

    DV_INL static Fp neg(const Fp& a) {
        Fp z = zero();
        return a.is_zero() ? a : sub(z, a);
    }

    DV_INL static Fp mul_inl(const Fp& a, const Fp& b) {
        uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t bi = b.v[i];
            asm("mad.lo.cc.u32 %0, %9, %13, %0;\n\t"
                "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"
                "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"
                "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"
                "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
                "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"
                "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"
                "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"
                "addc.u32 %8, %8, 0;"
                : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
                : "r"(a.v[0]), "r"(a.v[2]), "r"(a.v[4]), "r"(a.v[6]), "r"(bi));
            asm("mad.lo.cc.u32 %0, %8, %12, %0;\n\t"
                "madc.hi.cc.u32 %1, %8, %12, %1;\n\t"
                "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"
                "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
                "madc.lo.cc.u32 %4, %10, %12, %4;\n\t"
                "madc.hi.cc.u32 %5, %10, %12, %5;\n\t"
                "madc.lo.cc.u32 %6, %11, %12, %6;\n\t"
                "madc.hi.u32 %7, %11, %12, %7;"
                : "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
                : "r"(a.v[1]), "r"(a.v[3]), "r"(a.v[5]), "r"(a.v[7]), "r"(bi));
            const uint32_t m = t0 * C::INV;
            asm("mad.lo.cc.u32 %0, %9, %10, %0;\n\t"
                "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"
                "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"
                "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"
                "madc.lo.cc.u32 %4, %9, %12, %4;\n\t"
                "madc.hi.cc.u32 %5, %9, %12, %5;\n\t"
                "madc.lo.cc.u32 %6, %9, %13, %6;\n\t"
                "madc.hi.cc.u32 %7, %9, %13, %7;\n\t"
                "addc.u32 %8, %8, 0;"
                : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
                : "r"(m), "n"(C::P0), "n"(C::P2), "n"(C::P4), "n"(C::P6));
            asm("mad.lo.cc.u32 %0, %8, %9, %0;\n\t"
                "madc.hi.cc.u32 %1, %8, %9, %1;\n\t"
                "madc.lo.cc.u32 %2, %8, %10, %2;\n\t"
                "madc.hi.cc.u32 %3, %8, %10, %3;\n\t"
                "madc.lo.cc.u32 %4, %8, %11, %4;\n\t"
                "madc.hi.cc.u32 %5, %8, %11, %5;\n\t"
                "madc.lo.cc.u32 %6, %8, %12, %6;\n\t"
                "madc.hi.u32 %7, %8, %12, %7;"
                : "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
                : "r"(m), "n"(C::P1), "n"(C::P3), "n"(C::P5), "n"(C::P7));
            // t0 is now 0 (mod 2^32): shift one limb down.
            t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = t7; t7 = t8; t8 = 0;
        }
        Fp r;
        r.v[0] = t0; r.v[1] = t1; r.v[2] = t2; r.v[3] = t3;
        r.v[4] = t4; r.v[5] = t5; r.v[6] = t6; r.v[7] = t7;
        reduce_once(r.v);
        return r;
    }

    // One out-of-line copy of the multiplication keeps the point-arithmetic
    // loops inside the instruction cache (measured faster than inlining ten
    // ~300-instruction bodies per XYZZ addition).
#ifndef DV_MUL_INLINE
    __device__ __noinline__ static Fp mul(Fp a, Fp b) { return mul_inl(a, b); }
#else
    DV_INL static Fp mul(const Fp& a, const Fp& b) { return mul_inl(a, b); }
#endif
    // Two independent products in one out-of-line body: the compiler
    // interleaves their carry chains, which hides the multiply latency that a
    // lone chain exposes when few warps are resident.
    typedef PairOf<Fp> Pair;
#ifndef DV_MUL_INLINE
    __device__ __noinline__ static Pair mul2(Fp a, Fp b, Fp c, Fp d) { return {mul_inl(a, b), mul_inl(c, d)}; }
#else
    DV_INL static Pair mul2(const Fp& a, const Fp& b, const Fp& c, const Fp& d) {
        return {mul_inl(a, b), mul_inl(c, d)};
    }
#endif
    // Montgomery square: the cross products a_i a_j (i < j) once, summed by
    // columns in a three-word accumulator, doubled by a one-bit shift, plus
    // the diagonal a_i^2 in one carry chain; then eight word-by-word
    // reduction steps over the 512-bit square (two interleaved carry chains
    // per step as in mul_inl, e carrying into the word above the window).
    // 36 + 72 word products against a product's 136.
    DV_INL static Fp sqr_inl(const Fp& a) {
        uint32_t t[16];
        uint32_t c0 = 0, c1 = 0, c2 = 0;
        t[0] = 0;
#pragma unroll
        for (int k = 1; k < 14; ++k) {
#pragma unroll
            for (int i = (k > 7 ? k - 7 : 0); 2 * i < k; ++i)
                asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
                    "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
                    "addc.u32 %2, %2, 0;"
                    : "+r"(c0), "+r"(c1), "+r"(c2)
                    : "r"(a.v[i]), "r"(a.v[k - i]));
            t[k] = c0;
            c0 = c1;
            c1 = c2;
            c2 = 0;
        }
        t[14] = c0;
        t[15] = c1;
#pragma unroll
        for (int k = 15; k > 0; --k) t[k] = __funnelshift_l(t[k - 1], t[k], 1);
        asm("mad.lo.cc.u32 %0, %16, %16, %0;\n\t"
            "madc.hi.cc.u32 %1, %16, %16, %1;\n\t"
            "madc.lo.cc.u32 %2, %17, %17, %2;\n\t"
            "madc.hi.cc.u32 %3, %17, %17, %3;\n\t"
            "madc.lo.cc.u32 %4, %18, %18, %4;\n\t"
            "madc.hi.cc.u32 %5, %18, %18, %5;\n\t"
            "madc.lo.cc.u32 %6, %19, %19, %6;\n\t"
            "madc.hi.cc.u32 %7, %19, %19, %7;\n\t"
            "madc.lo.cc.u32 %8, %20, %20, %8;\n\t"
            "madc.hi.cc.u32 %9, %20, %20, %9;\n\t"
            "madc.lo.cc.u32 %10, %21, %21, %10;\n\t"
            "madc.hi.cc.u32 %11, %21, %21, %11;\n\t"
            "madc.lo.cc.u32 %12, %22, %22, %12;\n\t"
            "madc.hi.cc.u32 %13, %22, %22, %13;\n\t"
            "madc.lo.cc.u32 %14, %23, %23, %14;\n\t"
            "madc.hi.u32 %15, %23, %23, %15;"
            : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
              "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12]), "+r"(t[13]), "+r"(t[14]), "+r"(t[15])
            : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
              "r"(a.v[7]));
        uint32_t e = 0;  // carry into t[i + 8] at step i
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t m = t[i] * C::INV;
            asm("mad.lo.cc.u32 %0, %10, %11, %0;\n\t"
                "madc.hi.cc.u32 %1, %10, %11, %1;\n\t"
                "madc.lo.cc.u32 %2, %10, %12, %2;\n\t"
                "madc.hi.cc.u32 %3, %10, %12, %3;\n\t"
                "madc.lo.cc.u32 %4, %10, %13, %4;\n\t"
                "madc.hi.cc.u32 %5, %10, %13, %5;\n\t"
                "madc.lo.cc.u32 %6, %10, %14, %6;\n\t"
                "madc.hi.cc.u32 %7, %10, %14, %7;\n\t"
                "addc.cc.u32 %8, %8, %9;\n\t"
                "addc.u32 %9, 0, 0;"
                : "+r"(t[i]), "+r"(t[i + 1]), "+r"(t[i + 2]), "+r"(t[i + 3]), "+r"(t[i + 4]), "+r"(t[i + 5]),
                  "+r"(t[i + 6]), "+r"(t[i + 7]), "+r"(t[i + 8]), "+r"(e)
                : "r"(m), "n"(C::P0), "n"(C::P2), "n"(C::P4), "n"(C::P6));
            asm("mad.lo.cc.u32 %0, %9, %10, %0;\n\t"
                "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"
                "madc.lo.cc.u32 %2, %9, %11, %2;\n\t"
                "madc.hi.cc.u32 %3, %9, %11, %3;\n\t"
                "madc.lo.cc.u32 %4, %9, %12, %4;\n\t"
                "madc.hi.cc.u32 %5, %9, %12, %5;\n\t"
                "madc.lo.cc.u32 %6, %9, %13, %6;\n\t"
                "madc.hi.cc.u32 %7, %9, %13, %7;\n\t"
                "addc.u32 %8, %8, 0;"
                : "+r"(t[i + 1]), "+r"(t[i + 2]), "+r"(t[i + 3]), "+r"(t[i + 4]), "+r"(t[i + 5]), "+r"(t[i + 6]),
                  "+r"(t[i + 7]), "+r"(t[i + 8]), "+r"(e)
                : "r"(m), "n"(C::P1), "n"(C::P3), "n"(C::P5), "n"(C::P7));
        }
        Fp r;
#pragma unroll
        for (int j = 0; j < 8; ++j) r.v[j] = t[8 + j];
        reduce_once(r.v);
        return r;
    }
#ifndef DV_MUL_INLINE
    __device__ __noinline__ static Fp sqr(Fp a) { return sqr_inl(a); }
    // two independent squares in one body, like mul2
    __device__ __noinline__ static Pair sqr2(Fp a, Fp b) { return {sqr_inl(a), sqr_inl(b)}; }
#else
    DV_INL static Fp sqr(const Fp& a) { return sqr_inl(a); }
    DV_INL static Pair sqr2(const Fp& a, const Fp& b) { return {sqr_inl(a), sqr_inl(b)}; }
#endif

    // Canonical little-endian limbs <-> Montgomery form.
    DV_INL static Fp from_canonical(const uint32_t* c) {
        Fp a;
#pragma unroll
        for (int i = 0; i < 8; ++i) a.v[i] = c[i];
        return mul(a, r2());
    }
    DV_INL void to_canonical(uint32_t* c) const {
        Fp one_raw = zero();
        one_raw.v[0] = 1;
        Fp r = mul(*this, one_raw);
#pragma unroll
        for (int i = 0; i < 8; ++i) c[i] = r.v[i];
    }
    // Canonical check: c < p.
    DV_INL static bool is_canonical(const uint32_t* c) {
        const uint32_t p[8] = {C::P0, C::P1, C::P2, C::P3, C::P4, C::P5, C::P6, C::P7};
#pragma unroll
        for (int i = 7; i >= 0; --i) {
            if (c[i] < p[i]) return true;
            if (c[i] > p[i]) return false;
        }
        return false;
    }

    // a^e for a 256-bit exponent given as 8 little-endian limbs.
    DV_INL static Fp pow(const Fp& a, const uint32_t* e) {
        Fp r = one();
        for (int i = 255; i >= 0; --i) {
            r = sqr(r);
            if ((e[i >> 5] >> (i & 31)) & 1) r = mul(r, a);
        }
        return r;
    }
    // 1 / a (0 for a = 0) by the divsteps of Bernstein and Yang ("Fast
    // constant-time gcd computation and modular inversion", TCHES 2019),
    // run variable-time: with f = p, g = aR, d = 0, e = 1 (f = d aR and
    // g = e aR mod p throughout), each batch takes 30 divsteps on the low 30
    // bits of f and g into a transition matrix scaled by 2^30, then applies
    // it to f, g (exact division by 2^30) and to d, e (division by 2^30 mod
    // p, adding md p with md = -(u d + v e) p^-1 mod 2^30).  Numbers are 9
    // limbs of 30 bits, the top one signed.  736 divsteps bring g to 0 for
    // inputs below 2^254, so 25 batches bound the loop, which ends when
    // g = 0.  Then f = +-1 and (aR)^-1 = f d with |d| < 26 p; the
    // Montgomery product with R^3 mod p turns (aR)^-1 into a^-1 R.
    DV_INL static Fp inv(const Fp& a) {
        constexpr uint32_t M30 = (1u << 30) - 1;
        constexpr uint32_t PINV30 = (0u - C::INV) & M30;  // p^-1 mod 2^30
        N9 f, g, d, e;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            f.l[i] = limb30(i);
            d.l[i] = 0;
            e.l[i] = i == 0;
            g.l[i] = (int32_t)(bits30(a, i));
        }
        int delta = 1;
#pragma unroll 1
        for (int batch = 0; batch < 25 && g.nonzero(); ++batch) {
            int32_t t[4];
            delta = divsteps30(delta, (uint32_t)f.l[0], (uint32_t)g.l[0], t);
            // (f, g) <- t (f, g) / 2^30 exactly; (d, e) <- t (d, e) / 2^30 mod p
            int64_t cf = (int64_t)t[0] * f.l[0] + (int64_t)t[1] * g.l[0];
            int64_t cg = (int64_t)t[2] * f.l[0] + (int64_t)t[3] * g.l[0];
            int64_t cd = (int64_t)t[0] * d.l[0] + (int64_t)t[1] * e.l[0];
            int64_t ce = (int64_t)t[2] * d.l[0] + (int64_t)t[3] * e.l[0];
            const int32_t md = (int32_t)((0u - (uint32_t)cd * PINV30) & M30);
            const int32_t me = (int32_t)((0u - (uint32_t)ce * PINV30) & M30);
            cd += (int64_t)md * limb30(0);
            ce += (int64_t)me * limb30(0);
            cf >>= 30;
            cg >>= 30;
            cd >>= 30;
            ce >>= 30;
#pragma unroll
            for (int i = 1; i < 9; ++i) {
                cf += (int64_t)t[0] * f.l[i] + (int64_t)t[1] * g.l[i];
                cg += (int64_t)t[2] * f.l[i] + (int64_t)t[3] * g.l[i];
                cd += (int64_t)t[0] * d.l[i] + (int64_t)t[1] * e.l[i] + (int64_t)md * limb30(i);
                ce += (int64_t)t[2] * d.l[i] + (int64_t)t[3] * e.l[i] + (int64_t)me * limb30(i);
                f.l[i - 1] = (int32_t)((uint32_t)cf & M30);
                g.l[i - 1] = (int32_t)((uint32_t)cg & M30);
                d.l[i - 1] = (int32_t)((uint32_t)cd & M30);
                e.l[i - 1] = (int32_t)((uint32_t)ce & M30);
                cf >>= 30;
                cg >>= 30;
                cd >>= 30;
                ce >>= 30;
            }
            f.l[8] = (int32_t)cf;
            g.l[8] = (int32_t)cg;
            d.l[8] = (int32_t)cd;
            e.l[8] = (int32_t)ce;
        }
        // x = 32 p + f d in (6 p, 58 p), then conditional subtractions of 32 p .. p
        const bool neg = f.l[8] < 0;
        N9 x;
        int64_t c = 0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            c += 32 * (int64_t)limb30(i) + (neg ? -(int64_t)d.l[i] : (int64_t)d.l[i]);
            x.l[i] = i < 8 ? (int32_t)((uint32_t)c & M30) : (int32_t)c;
            c >>= 30;
        }
#pragma unroll
        for (int k = 5; k >= 0; --k) {
            N9 y;
            int64_t cy = 0;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                cy += (int64_t)x.l[i] - ((int64_t)limb30(i) << k);
                y.l[i] = i < 8 ? (int32_t)((uint32_t)cy & M30) : (int32_t)cy;
                cy >>= 30;
            }
            if (y.l[8] >= 0) x = y;
        }
        Fp r, r3;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            // bits [32 w, 32 w + 32) of x; 32 w mod 30 <= 14
            const int i = 32 * w / 30, s = 32 * w % 30;
            r.v[w] = ((uint32_t)x.l[i] >> s) | ((uint32_t)x.l[i + 1] << (30 - s));
        }
        r3.v[0] = C::R30; r3.v[1] = C::R31; r3.v[2] = C::R32; r3.v[3] = C::R33;
        r3.v[4] = C::R34; r3.v[5] = C::R35; r3.v[6] = C::R36; r3.v[7] = C::R37;
        return mul(r, r3);
    }

  private:
    // Signed 30-bit-limb numbers of the divstep inverse.
    struct N9 {
        int32_t l[9];
        DV_INL bool nonzero() const {
            int32_t o = 0;
#pragma unroll
            for (int i = 0; i < 9; ++i) o |= l[i];
            return o != 0;
        }
    };
    // bits [30 i, 30 i + 30) of p and of a
    DV_INL static constexpr int32_t limb30(int i) {
        const uint32_t p[8] = {C::P0, C::P1, C::P2, C::P3, C::P4, C::P5, C::P6, C::P7};
        const int b = 30 * i, w = b >> 5, s = b & 31;
        const uint32_t lo = p[w] >> s, hi = (s > 2 && w + 1 < 8) ? p[w + 1] << (32 - s) : 0u;
        return (int32_t)((lo | hi) & ((1u << 30) - 1));
    }
    DV_INL static uint32_t bits30(const Fp& a, int i) {
        const int b = 30 * i, w = b >> 5, s = b & 31;
        uint32_t x = a.v[w] >> s;
        if (s > 2 && w + 1 < 8) x |= a.v[w + 1] << (32 - s);
        return x & ((1u << 30) - 1);
    }
    // 30 divsteps on the low bits of f and g (f odd): delta and the matrix
    // t = (u, v, q, r) with t (f, g) = 2^30 (f', g').  A step with g odd and
    // delta > 0 swaps first: (f, g) <- (g, -f), (u, v, q, r) <- (q, r, -u, -v),
    // delta <- -delta; then g odd adds f to g and (u, v) to (q, r); then g
    // halves, (u, v) double and delta grows by one.
    DV_INL static int divsteps30(int delta, uint32_t f, uint32_t g, int32_t* t) {
        int32_t u = 1, v = 0, q = 0, r = 1;
#pragma unroll
        for (int i = 0; i < 30; ++i) {
            const bool odd = g & 1u, swap = odd && delta > 0;
            const uint32_t f1 = swap ? g : f, g1 = swap ? 0u - f : g;
            const int32_t u1 = swap ? q : u, v1 = swap ? r : v, q1 = swap ? -u : q, r1 = swap ? -v : r;
            delta = swap ? -delta : delta;
            f = f1;
            g = (odd ? g1 + f1 : g1) >> 1;
            q = odd ? q1 + u1 : q1;
            r = odd ? r1 + v1 : r1;
            u = 2 * u1;
            v = 2 * v1;
            ++delta;
        }
        t[0] = u;
        t[1] = v;
        t[2] = q;
        t[3] = r;
        return delta;
    }
};

typedef Fp<FqCfg> Fq;
typedef Fp<FrCfg> Fr;

// Fq2 = Fq[u] / (u^2 + 1)
struct Fq2 {
    Fq c0, c1;
    DV_INL static Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
    DV_INL static Fq2 one() { return {Fq::one(), Fq::zero()}; }
    DV_INL bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
    DV_INL bool operator==(const Fq2& o) const { return c0 == o.c0 && c1 == o.c1; }
    DV_INL static Fq2 add(const Fq2& a, const Fq2& b) { return {Fq::add(a.c0, b.c0), Fq::add(a.c1, b.c1)}; }
    DV_INL static Fq2 sub(const Fq2& a, const Fq2& b) { return {Fq::sub(a.c0, b.c0), Fq::sub(a.c1, b.c1)}; }
    DV_INL static Fq2 dbl(const Fq2& a) { return {Fq::dbl(a.c0), Fq::dbl(a.c1)}; }
    DV_INL static Fq2 neg(const Fq2& a) { return {Fq::neg(a.c0), Fq::neg(a.c1)}; }
    DV_INL static Fq2 conj(const Fq2& a) { return {a.c0, Fq::neg(a.c1)}; }
    DV_INL static Fq2 mul(const Fq2& a, const Fq2& b) {
        // Karatsuba: 3 base multiplications.
        const Fq t0 = Fq::mul(a.c0, b.c0);
        const Fq t1 = Fq::mul(a.c1, b.c1);
        const Fq t2 = Fq::mul(Fq::add(a.c0, a.c1), Fq::add(b.c0, b.c1));
        return {Fq::sub(t0, t1), Fq::sub(Fq::sub(t2, t0), t1)};
    }
    DV_INL static PairOf<Fq2> mul2(const Fq2& a, const Fq2& b, const Fq2& c, const Fq2& d) {
        return {mul(a, b), mul(c, d)};
    }
    DV_INL static Fq2 sqr(const Fq2& a) {
        // (c0 + c1 u)^2 = (c0+c1)(c0-c1) + 2 c0 c1 u
        const Fq m = Fq::mul(Fq::add(a.c0, a.c1), Fq::sub(a.c0, a.c1));
        const Fq c = Fq::mul(a.c0, a.c1);
        return {m, Fq::dbl(c)};
    }
    DV_INL static Fq2 mul_fq(const Fq2& a, const Fq& s) { return {Fq::mul(a.c0, s), Fq::mul(a.c1, s)}; }
    DV_INL static Fq2 inv(const Fq2& a) {
        const Fq n = Fq::add(Fq::sqr(a.c0), Fq::sqr(a.c1));
        const Fq ni = Fq::inv(n);
        return {Fq::mul(a.c0, ni), Fq::neg(Fq::mul(a.c1, ni))};
    }
};

}  // namespace dv
