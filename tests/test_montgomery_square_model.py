"""The limb schedule of the device Montgomery square (Fp::sqr_inl in
zkp-dynaverse_b200/csrc/field.cuh), restated step by step with PTX carry
semantics (mad.lo.cc / madc.hi.cc / addc) and checked against a^2 R^-1 mod p
for both BN254 fields.  The kernel relies on three bounds that the restatement
asserts: the cross-product sum fits 16 words after doubling, the word
reduced at each step becomes zero, and the carry word e stays at most 2
and ends at 0 (the result is below 2p < 2^256).  The device code itself is
covered by every GPU parity test."""
import random

M32 = (1 << 32) - 1
Q = 21888242871839275222246405745257275088696311157297823662689037894645226208583
R = 21888242871839275222246405745257275088548364400416034343698204186575808495617


def _limbs(x):
    return [(x >> (32 * i)) & M32 for i in range(8)]


def _mad(acc, x, y, lo, carry):
    """acc + lo/hi word of x * y + carry -> (word, carry out)."""
    prod = x * y
    s = acc + ((prod & M32) if lo else (prod >> 32)) + carry
    return s & M32, s >> 32


def sqr_model(a, p):
    inv = (-pow(p, -1, 1 << 32)) % (1 << 32)
    P = _limbs(p)
    t = [0] * 16
    c0 = c1 = c2 = 0
    for k in range(1, 14):  # columns of the cross products a_i a_j, i < j
        i = max(0, k - 7)
        while 2 * i < k:
            c0, cf = _mad(c0, a[i], a[k - i], True, 0)
            c1, cf = _mad(c1, a[i], a[k - i], False, cf)
            c2 = (c2 + cf) & M32
            i += 1
        t[k] = c0
        c0, c1, c2 = c1, c2, 0
    t[14], t[15] = c0, c1
    assert t[15] >> 31 == 0  # doubling keeps 16 words
    for k in range(15, 0, -1):  # __funnelshift_l(t[k-1], t[k], 1)
        t[k] = ((t[k] << 1) | (t[k - 1] >> 31)) & M32
    cf = 0
    for j in range(8):  # diagonal a_j^2, one carry chain
        t[2 * j], cf = _mad(t[2 * j], a[j], a[j], True, cf)
        t[2 * j + 1], cf = _mad(t[2 * j + 1], a[j], a[j], False, cf)
    assert cf == 0
    e = 0  # carry into t[i + 8] at step i
    for i in range(8):
        m = (t[i] * inv) & M32
        cf = 0
        for q, pj in enumerate((P[0], P[2], P[4], P[6])):
            t[i + 2 * q], cf = _mad(t[i + 2 * q], m, pj, True, cf)
            t[i + 2 * q + 1], cf = _mad(t[i + 2 * q + 1], m, pj, False, cf)
        s = t[i + 8] + e + cf
        t[i + 8], e = s & M32, s >> 32
        cf = 0
        for q, pj in enumerate((P[1], P[3], P[5], P[7])):
            t[i + 1 + 2 * q], cf = _mad(t[i + 1 + 2 * q], m, pj, True, cf)
            t[i + 2 + 2 * q], cf = _mad(t[i + 2 + 2 * q], m, pj, False, cf)
        e += cf
        assert t[i] == 0 and e <= 2
    assert e == 0
    r = sum(t[8 + j] << (32 * j) for j in range(8))
    return r - p if r >= p else r  # reduce_once


def test_square_schedule_matches_montgomery_square():
    rng = random.Random(5)
    for p in (Q, R):
        r_inv = pow(1 << 256, -1, p)
        cases = [0, 1, 2, p - 1, p - 2, (1 << 255) % p, (1 << 254) % p] + [rng.randrange(p) for _ in range(3000)]
        for x in cases:
            assert sqr_model(_limbs(x), p) == x * x * r_inv % p, hex(x)
