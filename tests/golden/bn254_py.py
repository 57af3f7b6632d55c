"""Pure-Python BN254 arithmetic used only to generate and check golden vectors.

Test infrastructure, not product code.  Everything here is written with
Python's arbitrary-precision integers and plain affine formulas, so it shares
no code (and no Montgomery machinery) with either the C oracle or the CUDA
kernels.  It restates the published arithmetic that the reference reaches
through arkworks 0.4 (ark-bn254 0.4.0 curve constants, ark-ff 0.4.2 field
semantics, ark-poly 0.4.2 Radix2EvaluationDomain):

* Fr NTT semantics: crates/gpu/src/lib.rs:99-118 (CpuBackend::ntt) and
  crates/protocol/src/dynaverse.rs:1157-1164 (ArkReferenceBackend::ntt).
* Root orientation: crates/gpu/src/icicle.rs:440-443 passes
  Fr::get_root_of_unity(2^20); ark-ff derives it from TWO_ADIC_ROOT_OF_UNITY
  = GENERATOR^((r-1)/2^28) with GENERATOR = 5 by repeated squaring.
* G2 subgroup predicates: crates/gpu/src/g2_validation.rs:250-299.
* G2 wire parsing: native/include/icicle_g2_wire.cuh:17-32 and
  crates/gpu/src/g2_validation.rs:243-248.
"""

Q = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
FR_GENERATOR = 5
TWO_ADICITY = 28
BN_SEED = 4965661367192848881

G1_GEN = (1, 2)
G2_GEN = (
    (10857046999023057135944570762232829481370756359578518086990519993285655852781,
     11559732032986387107991004021392285783925812861821192530917403151452391805634),
    (8495653923123431417604973247489272438418190587263600148770280649306958101930,
     4082367875863433681332203403145435568316851327593401208105741076214120093531),
)


# ---------------------------------------------------------------- ChaCha20
def _rotl(v, c):
    return ((v << c) & 0xFFFFFFFF) | (v >> (32 - c))


def _quarter(s, a, b, c, d):
    s[a] = (s[a] + s[b]) & 0xFFFFFFFF; s[d] = _rotl(s[d] ^ s[a], 16)
    s[c] = (s[c] + s[d]) & 0xFFFFFFFF; s[b] = _rotl(s[b] ^ s[c], 12)
    s[a] = (s[a] + s[b]) & 0xFFFFFFFF; s[d] = _rotl(s[d] ^ s[a], 8)
    s[c] = (s[c] + s[d]) & 0xFFFFFFFF; s[b] = _rotl(s[b] ^ s[c], 7)


def chacha20_block(key_words, counter, nonce_words=(0, 0, 0)):
    """RFC 8439 block function; returns 64 bytes."""
    init = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(key_words) + \
        [counter & 0xFFFFFFFF] + list(nonce_words)
    s = list(init)
    for _ in range(10):
        _quarter(s, 0, 4, 8, 12); _quarter(s, 1, 5, 9, 13)
        _quarter(s, 2, 6, 10, 14); _quarter(s, 3, 7, 11, 15)
        _quarter(s, 0, 5, 10, 15); _quarter(s, 1, 6, 11, 12)
        _quarter(s, 2, 7, 8, 13); _quarter(s, 3, 4, 9, 14)
    out = bytearray()
    for i in range(16):
        out += ((s[i] + init[i]) & 0xFFFFFFFF).to_bytes(4, "little")
    return bytes(out)


class ChaCha20Stream:
    """Seeded stream: key = seed (u64 LE) followed by 24 zero bytes, nonce 0."""

    def __init__(self, seed):
        key = seed.to_bytes(8, "little") + bytes(24)
        self.key_words = [int.from_bytes(key[4 * i:4 * i + 4], "little") for i in range(8)]
        self.counter = 0
        self.buf = b""

    def read(self, n):
        while len(self.buf) < n:
            self.buf += chacha20_block(self.key_words, self.counter)
            self.counter += 1
        out, self.buf = self.buf[:n], self.buf[n:]
        return out

    def uniform(self, modulus):
        """Rejection sampling on 254-bit masked 32-byte words."""
        while True:
            v = int.from_bytes(self.read(32), "little") & ((1 << 254) - 1)
            if v < modulus:
                return v


# ---------------------------------------------------------------- fields
def inv(a, m=Q):
    return pow(a, -1, m)


def f2add(a, b): return ((a[0] + b[0]) % Q, (a[1] + b[1]) % Q)
def f2sub(a, b): return ((a[0] - b[0]) % Q, (a[1] - b[1]) % Q)
def f2neg(a): return ((-a[0]) % Q, (-a[1]) % Q)
def f2mul(a, b): return ((a[0] * b[0] - a[1] * b[1]) % Q, (a[0] * b[1] + a[1] * b[0]) % Q)


def f2inv(a):
    n = inv((a[0] * a[0] + a[1] * a[1]) % Q)
    return (a[0] * n % Q, (-a[1]) * n % Q)


def f2pow(a, e):
    out = (1, 0)
    while e:
        if e & 1:
            out = f2mul(out, a)
        a = f2mul(a, a)
        e >>= 1
    return out


def f2sqrt(a):
    """Square root in Fq2 = Fq[u]/(u^2+1) for q = 3 mod 4, or None."""
    if a == (0, 0):
        return (0, 0)
    a1 = f2pow(a, (Q - 3) // 4)
    alpha = f2mul(a1, f2mul(a1, a))
    a0 = f2mul(f2pow(alpha, Q), alpha)
    if a0 == (Q - 1, 0):
        return None
    x0 = f2mul(a1, a)
    if alpha == (Q - 1, 0):
        x = f2mul((0, 1), x0)
    else:
        b = f2pow(f2add((1, 0), alpha), (Q - 1) // 2)
        x = f2mul(b, x0)
    return x if f2mul(x, x) == a else None


B1 = 3
B2 = f2mul((3, 0), f2inv((9, 1)))


# ---------------------------------------------------------------- G1 affine
def g1_on_curve(p):
    return p is None or (p[1] * p[1] - p[0] ** 3 - B1) % Q == 0


def g1_add(p, s):
    if p is None:
        return s
    if s is None:
        return p
    if p[0] == s[0]:
        if (p[1] + s[1]) % Q == 0:
            return None
        lam = 3 * p[0] * p[0] * inv(2 * p[1]) % Q
    else:
        lam = (s[1] - p[1]) * inv((s[0] - p[0]) % Q) % Q
    x = (lam * lam - p[0] - s[0]) % Q
    return (x, (lam * (p[0] - x) - p[1]) % Q)


def g1_neg(p):
    return None if p is None else (p[0], (-p[1]) % Q)


def g1_mul(p, k):
    out = None
    while k:
        if k & 1:
            out = g1_add(out, p)
        p = g1_add(p, p)
        k >>= 1
    return out


# ---------------------------------------------------------------- G2 affine
def g2_on_curve(p):
    if p is None:
        return True
    x, y = p
    return f2sub(f2mul(y, y), f2add(f2mul(f2mul(x, x), x), B2)) == (0, 0)


def g2_add(p, s):
    if p is None:
        return s
    if s is None:
        return p
    if p[0] == s[0]:
        if f2add(p[1], s[1]) == (0, 0):
            return None
        lam = f2mul(f2mul((3, 0), f2mul(p[0], p[0])), f2inv(f2add(p[1], p[1])))
    else:
        lam = f2mul(f2sub(s[1], p[1]), f2inv(f2sub(s[0], p[0])))
    x = f2sub(f2sub(f2mul(lam, lam), p[0]), s[0])
    return (x, f2sub(f2mul(lam, f2sub(p[0], x)), p[1]))


def g2_neg(p):
    return None if p is None else (p[0], f2neg(p[1]))


def g2_mul(p, k):
    out = None
    while k:
        if k & 1:
            out = g2_add(out, p)
        p = g2_add(p, p)
        k >>= 1
    return out


PSI_CX = f2pow((9, 1), (Q - 1) // 3)
PSI_CY = f2pow((9, 1), (Q - 1) // 2)


def psi(p):
    if p is None:
        return None
    conj = lambda a: (a[0], (-a[1]) % Q)
    return (f2mul(conj(p[0]), PSI_CX), f2mul(conj(p[1]), PSI_CY))


def subgroup_full_order(p):
    return g2_mul(p, R) is None


def subgroup_frobenius_127(p):
    return psi(p) == g2_mul(p, 6 * BN_SEED * BN_SEED)


def subgroup_frobenius_63(p):
    a = g2_mul(p, BN_SEED)
    b = psi(a)
    c = psi(b)
    lhs = g2_add(g2_add(g2_add(a, p), b), c)
    d = psi(c)
    return lhs == g2_add(d, d)


def twist_point_from_x(x):
    """get_point_from_x_unchecked(x, greatest=false): smaller of the two roots
    in arkworks' Fq2 order (c1 compared first, then c0)."""
    y = f2sqrt(f2add(f2mul(f2mul(x, x), x), B2))
    if y is None:
        return None
    ny = f2neg(y)
    key = lambda a: (a[1], a[0])
    return (x, min(y, ny, key=key))


# ---------------------------------------------------------------- NTT
def root_of_unity(n):
    """ark-ff get_root_of_unity for n = 2^k: TWO_ADIC_ROOT_OF_UNITY squared
    (28 - k) times."""
    k = n.bit_length() - 1
    assert n == 1 << k and k <= TWO_ADICITY
    w = pow(FR_GENERATOR, (R - 1) >> TWO_ADICITY, R)
    for _ in range(TWO_ADICITY - k):
        w = w * w % R
    return w


def dft(values, inverse=False, coset=False):
    """Direct O(n^2) evaluation with arkworks' Radix2EvaluationDomain meaning:
    forward = evaluations at w^i of sum_j c_j X^j; inverse = coefficients
    (scaled by 1/n).  coset uses offset g = 5: forward evaluates at g*w^i,
    inverse undoes it."""
    n = len(values)
    w = root_of_unity(n)
    if inverse:
        w = inv(w, R)
    out = []
    for i in range(n):
        wi = pow(w, i, R)
        acc, pw = 0, 1
        for j in range(n):
            acc += values[j] * pw
            pw = pw * wi % R
        out.append(acc % R)
    if inverse:
        ninv = inv(n, R)
        out = [v * ninv % R for v in out]
        if coset:
            ginv = inv(FR_GENERATOR, R)
            out = [v * pow(ginv, i, R) % R for i, v in enumerate(out)]
        return out
    if coset:
        # forward coset: scale coefficient j by g^j first
        scaled = [values[j] * pow(FR_GENERATOR, j, R) % R for j in range(n)]
        return dft(scaled, inverse=False, coset=False)
    return out


# ---------------------------------------------------------------- codecs
def fe_bytes(v):
    return v.to_bytes(32, "little")


def g1_bytes(p):
    return bytes(64) if p is None else fe_bytes(p[0]) + fe_bytes(p[1])


def g2_bytes(p):
    if p is None:
        return bytes(128)
    return fe_bytes(p[0][0]) + fe_bytes(p[0][1]) + fe_bytes(p[1][0]) + fe_bytes(p[1][1])


def g2_wire_mask(b, predicate=subgroup_full_order):
    """Per-point failure mask: 1 encoding, 2 off-curve, 4 outside subgroup."""
    assert len(b) == 128
    if b == bytes(128):
        return 0
    flags = b[127] & 0xC0
    if flags == 0xC0:
        return 1
    fields = []
    for j in range(4):
        chunk = bytearray(b[32 * j:32 * j + 32])
        if j == 3:
            chunk[31] &= 0x3F
        v = int.from_bytes(chunk, "little")
        if v >= Q:
            return 1
        fields.append(v)
    if flags == 0x40:
        return 0
    p = ((fields[0], fields[1]), (fields[2], fields[3]))
    if not g2_on_curve(p):
        return 2
    return 0 if predicate(p) else 4


# ---------------------------------------------------------------- pairing
# The optimal ate pairing with plain Python integers, for pinning the
# oracle: Fq12 is the flat field Fq[w] / (w^12 - 18 w^6 + 82) (w^6 = xi =
# 9 + u, u^2 = -1), lists of 12 coefficients.  The twist point T stays in
# affine Fq2 coordinates; the line through T with slope lam, untwisted by
# (x, y) -> (x w^2, y w^3), evaluated at P = (xp, yp) is
#     yp - lam xp w + (lam xT - yT) w^3.
# Loop: the NAF of 6z + 2, then the lines to pi(Q) and -pi^2(Q).  Final
# exponentiation: (q^12 - 1)/r times 2z(6z^2 + 3z + 1) (the exponent of the
# Fuentes-Castaneda, Knapp and Rodriguez-Henriquez hard part).
F12_ONE = [1] + [0] * 11
FINAL_EXP_MULTIPLE = 2 * BN_SEED * (6 * BN_SEED ** 2 + 3 * BN_SEED + 1)


def f12mul(a, b):
    t = [0] * 23
    for i, x in enumerate(a):
        if x:
            for j, y in enumerate(b):
                t[i + j] += x * y
    for k in range(22, 11, -1):  # w^12 = 18 w^6 - 82
        c = t[k]
        if c:
            t[k - 6] += 18 * c
            t[k - 12] -= 82 * c
    return [v % Q for v in t[:12]]


def f12pow(a, e):
    out = F12_ONE
    while e:
        if e & 1:
            out = f12mul(out, a)
        a = f12mul(a, a)
        e >>= 1
    return out


def _f2_at(line, k, a):
    """line += a w^k for a in Fq2 (u = w^6 - 9)."""
    line[k] = (line[k] + a[0] - 9 * a[1]) % Q
    line[k + 6] = (line[k + 6] + a[1]) % Q


def _line(lam, t, p):
    out = [0] * 12
    out[0] = p[1] % Q
    _f2_at(out, 1, f2neg(f2mul(lam, (p[0], 0))))
    _f2_at(out, 3, f2sub(f2mul(lam, t[0]), t[1]))
    return out


def naf(k):
    digits = []
    while k:
        if k & 1:
            d = 2 - (k & 3)
            k -= d
        else:
            d = 0
        digits.append(d)
        k >>= 1
    return digits[::-1]  # most significant first


def miller_loop(p, q):
    if p is None or q is None:
        return F12_ONE
    t, f = q, F12_ONE
    for d in naf(6 * BN_SEED + 2)[1:]:
        lam = f2mul(f2mul((3, 0), f2mul(t[0], t[0])), f2inv(f2add(t[1], t[1])))
        f = f12mul(f12mul(f, f), _line(lam, t, p))
        t = g2_add(t, t)
        if d:
            s = q if d == 1 else g2_neg(q)
            lam = f2mul(f2sub(s[1], t[1]), f2inv(f2sub(s[0], t[0])))
            f = f12mul(f, _line(lam, t, p))
            t = g2_add(t, s)
    q1 = psi(q)
    q2 = g2_neg(psi(q1))
    for s in (q1, q2):
        lam = f2mul(f2sub(s[1], t[1]), f2inv(f2sub(s[0], t[0])))
        f = f12mul(f, _line(lam, t, p))
        t = g2_add(t, s)
    return f


def final_exponentiation(f):
    return f12pow(f, (Q ** 12 - 1) // R * FINAL_EXP_MULTIPLE)


def pairing(p, q):
    return final_exponentiation(miller_loop(p, q))


def gt_bytes(f):
    """Tower serialisation (c0.c0.c0, c0.c0.c1, c0.c1.c0, ..., c1.c2.c1), Fq12 =
    Fq6 + Fq6 w, Fq6 = Fq2 + Fq2 v + Fq2 v^2, v = w^2: the Fq2 coefficient of
    w^k is (f[k] + 9 f[k + 6], f[k + 6])."""
    out = b""
    for k in (0, 2, 4, 1, 3, 5):
        out += fe_bytes((f[k] + 9 * f[k + 6]) % Q) + fe_bytes(f[k + 6])
    return out
