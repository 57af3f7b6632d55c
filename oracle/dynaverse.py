"""CPU restatement of the Dynaverse proof system -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
arm may import this module; the CUDA library never does.

Restates, for the fan-in-two toy circuit (crates/protocol/src/toy_circuit.rs),
the reference's
  * setup from the two trapdoors: SharedSrs::setup_with_backend_traced
    (srs.rs:147-197), DynamoParams::from_trapdoors_with_backend
    (dynamo.rs:140-233), SliceConsistencyKey::setup_six / from_impl
    (consistency.rs:165-290), KzgParams::from_tau_with_backend
    (kzg.rs:107-127), SparseUpdateBases (srs.rs:56-122) and the verifying key
    (dynaverse.rs:104-147);
  * the anchor proof prove_anchor_traced (dynaverse.rs:149-248) and its
    opening cache precompute_anchor_openings (dynaverse.rs:300-311);
  * the fixed-anchor sparse delta proof prove_delta_sparse_traced
    (dynaverse/sparse.rs:79-276);
  * the session rules of UpdateSession::apply (dynaverse/session.rs:51-142),
    including the synchronous re-anchor (update_proof_backend,
    dynaverse.rs:379-470);
  * the verifier verify_traced in Product mode (dynaverse.rs:843-1120), as
    the pairing-product equations PairingChecks::equal submits
    (verification.rs:37-144).

Two independent routes compute every commitment:
  route "bases"  the reference's own steps: SRS points from the
                 trapdoor-derived scalars by fixed-base multiplication, then
                 sparse and dense MSMs over them, NTT interpolation, the
                 subproduct tree, FFT products, exact division -- the
                 group and polynomial work in the C++ oracle
                 (bn254_oracle.cpp);
  route "scalar" every commitment is [s]G for the scalar s that the same
                 linear combination takes at the trapdoors (an MSM over
                 bases [b_i]G is [sum v_i b_i]G; a commitment to a
                 polynomial p is [p(tau_x)]G), in Python integers, then one
                 fixed-base multiplication per point.  Fast enough for
                 n = 65536, where the bases route's setup is not.
tests/test_oracle_dynaverse.py checks that the routes agree byte for byte
and that the bases route meets the properties the reference's own tests
assert (sparse delta == dense delta, sparse bases == dense commitments,
cached openings == dense openings, session == update_proof, verifier
verdicts).

Proof bytes (no canonical serialisation exists in the reference, whose
proof types are Rust structs, types.rs:64-172): the fields in declaration
order, G1 64 B and G2 128 B in the wire format (codec.rs:25-111,
resident.rs:419-431, infinity all zero):
  AnchorProof   3968 B  wires s1..s6 | s5_g2 | w_commitment | h_commitment |
                        dynamo (alpha, beta, h, z, b, q, instance_z,
                        instance_h) | consistency 6 x (qac, qcd, qbd, d,
                        a_degree, b_degree, d_degree) | public_zero_quotient |
                        multiplication_quotient
  DeltaProof    5312 B  changed_wires s1..s6 | changed_w | changed_h | dynamo |
                        consistency | public_zero_quotient | affected_g1 |
                        affected_g2 | unaffected_g1 | unaffected_g2 |
                        anchor_local s4..s6 | changed_local s4..s6 |
                        updated_s5_g2 | anchor_openings s4..s6 |
                        changed_openings s4..s6 | unaffected_zero s4..s6 |
                        local_multiplication_quotient
  DynaverseProof 9304 B anchor | delta (zero when absent) | u64 has_delta |
                        u64 anchor_generation | u64 generation  (LE)
"""
import struct

from . import oracle as O

R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
Q = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
TWO_ADIC_ROOT = pow(5, (R - 1) >> 28, R)  # ark-bn254 Fr TWO_ADIC_ROOT_OF_UNITY
G1_ZERO = bytes(64)
G2_ZERO = bytes(128)
ANCHOR_BYTES = 3968
DELTA_BYTES = 5312
PROOF_BYTES = ANCHOR_BYTES + DELTA_BYTES + 24


# ------------------------------------------------------------------ field
def fr(x: int) -> bytes:
    return (x % R).to_bytes(32, "little")


def frs(xs) -> bytes:
    return b"".join((x % R).to_bytes(32, "little") for x in xs)


def to_int(b: bytes) -> int:
    return int.from_bytes(b, "little")


def ints(b: bytes):
    return [int.from_bytes(b[i:i + 32], "little") for i in range(0, len(b), 32)]


def inv(a: int) -> int:
    a %= R
    if a == 0:
        raise ZeroDivisionError("inverse of zero")
    return pow(a, R - 2, R)


def batch_inv(xs):
    """Montgomery's simultaneous inversion (ark_ff::batch_inversion)."""
    n = len(xs)
    pre = [1] * (n + 1)
    for i, x in enumerate(xs):
        if x % R == 0:
            raise ZeroDivisionError("inverse of zero")
        pre[i + 1] = pre[i] * x % R
    t = inv(pre[n]) if n else 1
    out = [0] * n
    for i in range(n - 1, -1, -1):
        out[i] = t * pre[i] % R
        t = t * xs[i] % R
    return out


def root_of_unity(size: int) -> int:
    """Fr::get_root_of_unity(size): TWO_ADIC_ROOT squared down (ark-ff 0.4)."""
    log = size.bit_length() - 1
    assert size == 1 << log and log <= 28
    return pow(TWO_ADIC_ROOT, 1 << (28 - log), R)


def powers(x: int, n: int):
    out, p = [0] * n, 1
    for i in range(n):
        out[i] = p
        p = p * x % R
    return out


def lagrange_values(tau: int, size: int):
    """L_i(tau) = (tau^s - 1) omega^i / (s (tau - omega^i)) (setup.rs:48-61)."""
    num = (pow(tau, size, R) - 1) % R
    if num == 0:
        raise ValueError("Lagrange evaluation point lies on domain")
    roots = powers(root_of_unity(size), size)
    dens = batch_inv([(tau - w) % R for w in roots])
    scale = num * inv(size) % R
    return [d * scale % R * w % R for d, w in zip(dens, roots)]


def ceil_sqrt(n: int) -> int:
    """dynaverse.rs:826-833."""
    root = 1
    while root < n // root or (root == n // root and n % root != 0):
        root += 1
    return root


def sigma(n: int, i: int) -> int:
    """ToyCircuit permutation (toy_circuit.rs:17-27): swaps i <-> 6n+i and
    2n+i <-> 3n+i for i < n; an involution, so it is its own inverse."""
    if i < n:
        return 6 * n + i
    if 6 * n <= i < 7 * n:
        return i - 6 * n
    if 2 * n <= i < 3 * n:
        return i + n
    if 3 * n <= i < 4 * n:
        return i - n
    return i


def valid_instance(n: int):
    """ToyCircuit::valid_instance (toy_circuit.rs:45-70)."""
    pub = [0] * n
    w = [0] * (6 * n)
    for i in range(n):
        left = 1 if i == 0 else i + 1
        right = R - 1 if i == 0 else 2 * i + 3
        s = (left + right) % R
        mul = i + 7
        pub[i] = left
        w[i], w[n + i], w[2 * n + i], w[3 * n + i] = left, right, s, s
        w[4 * n + i] = mul
        w[5 * n + i] = s * mul % R
    return pub, w


def check_gates(n, pub, w, gates):
    """ToyCircuit::validate restricted to `gates` (toy_circuit.rs:72-90,
    session.rs:75-80)."""
    for i in gates:
        if w[i] != pub[i]:
            raise ValueError(f"public copy constraint fails at {i}")
        if w[2 * n + i] != w[3 * n + i]:
            raise ValueError(f"wire copy constraint fails at {i}")
        if (w[i] + w[n + i]) % R != w[2 * n + i]:
            raise ValueError(f"addition gate fails at {i}")
        if w[3 * n + i] * w[4 * n + i] % R != w[5 * n + i]:
            raise ValueError(f"multiplication gate fails at {i}")


def canonicalize(indices, values, length):
    """Update::canonicalize (types.rs:27-55): sort, last value wins."""
    if len(indices) != len(values):
        raise ValueError("update indices/values length mismatch")
    out = {}
    for i, v in sorted(zip(indices, values), key=lambda p: p[0]):  # stable
        out[i] = v % R
    if out and max(out) >= length:
        raise ValueError("update index out of range")
    return out


def sample_trapdoors(seed: int, n: int):
    """Trapdoor pair satisfying the rejection rules of srs.rs:158-178,
    drawn from the oracle's seeded ChaCha20 stream."""
    m = 8 * n
    k = 0
    while True:
        a, b = ints(O.uniform_fr(seed * 1000 + k, 2))
        k += 1
        if a == 0 or b == 0 or pow(a, m, R) == 1 or pow(b, m, R) == 1 or a == b:
            continue
        if a == pow(b, 8, R):  # tau_x == lambda y^r with lambda = 1 (n-aligned slices)
            continue
        return a, b


# ------------------------------------------------------------------ group helpers
def g1_neg(p: bytes) -> bytes:
    if p == G1_ZERO:
        return p
    return p[:32] + ((Q - to_int(p[32:])) % Q).to_bytes(32, "little")


def g1_add(a: bytes, b: bytes) -> bytes:
    return O.g1_add(a, b)


def g1_sub(a: bytes, b: bytes) -> bytes:
    return O.g1_add(a, g1_neg(b))


def g1_of(scalars):
    """[s]G1 for each scalar (one fixed-base call)."""
    s = list(scalars)
    if not s:
        return []
    out = O.fixed_base_g1(frs(s))
    return [out[64 * i:64 * i + 64] for i in range(len(s))]


def g2_of(scalars):
    s = list(scalars)
    if not s:
        return []
    out = O.fixed_base_g2(frs(s))
    return [out[128 * i:128 * i + 128] for i in range(len(s))]


def g1_gen() -> bytes:
    return g1_of([1])[0]


def g2_gen() -> bytes:
    return g2_of([1])[0]


def eval_poly(coeffs, x):
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % R
    return acc


# ------------------------------------------------------------------ parameters
class Params:
    """DynaverseParams for ToyCircuit(n) from explicit trapdoors (the
    reference samples them in setup and discards them; the oracle keeps
    them).  The trapdoor-derived scalars of every base are computed for
    indices the proofs can touch: witness entries lie below 6n, their
    Dynamo h images below 7n (sigma maps [0, n) to [6n, 7n))."""

    def __init__(self, n: int, tau_x: int, tau_y: int, route: str = "scalar", threads: int = 0):
        assert n > 0 and n & (n - 1) == 0
        assert route in ("scalar", "bases")
        self.n, self.m, self.route, self.threads = n, 8 * n, route, threads
        m = self.m
        self.tx, self.ty = tau_x % R, tau_y % R
        tx, ty = self.tx, self.ty
        txm, tym = pow(tx, m, R), pow(ty, m, R)
        if tx == 0 or ty == 0 or txm == 1 or tym == 1 or tx == ty:
            raise ValueError("trapdoors must be nonzero, distinct and outside the domain")
        if tx == pow(ty, 8, R):
            raise ValueError("consistency divisor vanishes")
        self.txm, self.tym = txm, tym
        self.wm = root_of_unity(m)
        self.wn = root_of_unity(n)
        inv_m = inv(m)
        # Dynamo (dynamo.rs:170-205): lx, ly over the big domain.  u sums
        # lx_i y_i over all of it; y_i = ly_i - ly_sigma(i) vanishes where
        # sigma fixes i, so only [0, 4n) and [6n, 7n) contribute.
        big = 7 * n
        wm_pows = powers(self.wm, big)
        lx_scale = (txm - 1) * inv_m % R
        ly_scale = (tym - 1) * inv_m % R
        dx = batch_inv([(tx - w) % R for w in wm_pows])
        dy = batch_inv([(ty - w) % R for w in wm_pows])
        self.lx = [lx_scale * w % R * d % R for w, d in zip(wm_pows, dx)]
        self.ly = [ly_scale * w % R * d % R for w, d in zip(wm_pows, dy)]
        self.y = [(self.ly[i] - self.ly[sigma(n, i)]) % R for i in range(big)]
        u = 0
        for i in range(big):
            if self.y[i]:
                u = (u + self.lx[i] * self.y[i]) % R
        self.u = u
        xv_inv = inv(txm - 1)
        tx_inv = inv(tx)
        self.alpha = [self.lx[i] * (u - self.y[i]) % R * xv_inv % R for i in range(big)]
        common = [self.y[i] * (self.lx[i] - inv_m) % R for i in range(big)]
        self.beta = [c * tx_inv % R for c in common]
        self.zb = [tym * l % R for l in self.lx]
        self.hb = [txm * y % R for y in self.y]
        self.bb = [c * tx % R for c in common]
        # consistency (consistency.rs:165-290); lambda = 1 for n-aligned slices
        ratio = m // n
        self.lsx = lagrange_values(tx, n)  # also SparseUpdateBases::small_lagrange (srs.rs:72-82)
        self.cx = lagrange_values(pow(tx, ratio, R), n)
        self.cy = lagrange_values(pow(ty, ratio, R), n)
        self.z_in = []
        for t in range(6):
            z = 1
            for i in range(t * n, (t + 1) * n):
                z = z * (tx - wm_pows[i]) % R
            self.z_in.append(z)
        z_in_inv = [inv(z) for z in self.z_in]
        six = 6 * n
        self.qac = []
        for t in range(6):
            col = []
            for i in range(six):
                mapped = self.cx[i - t * n] if t * n <= i < (t + 1) * n else 0
                col.append((self.lx[i] - mapped) * z_in_inv[t] % R)
            self.qac.append(col)
        xy_inv = inv(tx - ty)
        sub_inv = inv(tx - pow(ty, ratio, R))
        self.qcd = [(self.cx[j] - self.cy[j]) * xy_inv % R for j in range(n)]
        self.qbd = [(self.lsx[j] - self.cy[j]) * sub_inv % R for j in range(n)]
        self.dd = list(self.cy)
        self.adeg = [l * tym % R for l in self.lx[:six]]
        self.bdeg = [l * tym % R for l in self.lsx]
        self.ddeg = [c * txm % R for c in self.cy]
        # sparse update bases (srs.rs:56-122)
        self.small_points = powers(self.wn, n)
        small_inv = batch_inv([(tx - x) % R for x in self.small_points])
        self.open_u = [(self.lsx[j] - 1) * small_inv[j] % R for j in range(n)]
        ix = 1
        w = pow(self.wm, six, R)
        for _ in range(six, m):
            ix = ix * (tx - w) % R
            w = w * self.wm % R
        self.ix = ix  # I_x(tau_x), I_x vanishing on the public roots [6n, m)
        ix_inv = inv(ix)
        self.pq = [l * ix_inv % R for l in self.lx[:six]]
        self.public_h = [(self.ly[six + k] - self.ly[k]) % R for k in range(n)]  # dynamo.rs:112-124
        self.zn = (pow(tx, n, R) - 1) % R  # X^n - 1 at tau_x
        self.rebuild_interval = ceil_sqrt(n)
        self.g1 = g1_gen()
        self.g2 = g2_gen()
        # verifying key (dynaverse.rs:120-145, dynamo.rs:207-215, consistency.rs:267-273)
        vk = g2_of([u, tx, tx * tx, txm, tym, inv_m, txm - 1, tym - 1,
                    (tx - ty), (tx - pow(ty, ratio, R)), self.ix, self.zn] + self.z_in)
        self.vk_u, self.vk_x, self.vk_x2, self.vk_xm, self.vk_ym, self.vk_inv_m = vk[:6]
        self.vk_xm1, self.vk_ym1 = vk[6], vk[7]
        self.vk_x_minus_y, self.vk_x_minus_ly = vk[8], vk[9]
        self.public_zero_divisor, self.multiplication_divisor = vk[10], vk[11]
        self.vk_z_in = vk[12:18]
        self.multiplication_vanishing_g1 = g1_of([self.zn])[0]
        self.public_h_bases = g1_of(self.public_h)
        if route == "bases":
            self._build_bases()

    # ------------------------------------------------------------ bases route setup
    def _build_bases(self):
        """SRS points from the base scalars (setup.rs:13-31).  The reference's
        dense families span the big domain m, but a witness is zero from 6n
        on and its Dynamo h from 7n on, so every MSM of a proof touches only
        the families' first 6n (7n for ly) bases: those are built.  The KZG
        G1 powers span m (the anchor commits the m interpolation
        coefficients of the padded witness); G2 commitments span at most n + 1."""
        n, m = self.n, self.m
        th = self.threads
        f1 = lambda s: _split(O.fixed_base_g1(frs(s), th), 64)
        six = 6 * n
        self.B = {}
        self.B["lx"] = f1(self.lx[:six])
        self.B["ly"] = f1(self.ly)
        self.B["alpha"] = f1(self.alpha[:six])
        self.B["beta"] = f1(self.beta[:six])
        self.B["z"] = f1(self.zb[:six])
        self.B["h"] = f1(self.hb[:six])
        self.B["b"] = f1(self.bb[:six])
        for t in range(6):
            self.B[f"qac{t}"] = f1(self.qac[t])
        self.B["qcd"] = f1(self.qcd)
        self.B["qbd"] = f1(self.qbd)
        self.B["d"] = f1(self.dd)
        self.B["adeg"] = f1(self.adeg)
        self.B["bdeg"] = f1(self.bdeg)
        self.B["ddeg"] = f1(self.ddeg)
        self.B["lag"] = f1(self.lsx)
        self.B["open_u"] = f1(self.open_u)
        self.B["pq"] = f1(self.pq)
        self.kzg_g1 = O.fixed_base_g1(O.fr_powers(fr(self.tx), m), th)
        self.kzg_g2 = O.fixed_base_g2(O.fr_powers(fr(self.tx), 2 * n), th)  # A has up to n + 1 coefficients
        self.lag_g2 = _split(O.fixed_base_g2(frs(self.lsx), th), 128)
        self._prepared = None  # G1 transform of the powers for the opening cache (kzg.rs:248-275)

    # ------------------------------------------------------------ shared helpers
    def h_sparse(self, entries):
        """derive_h_sparse (dynamo.rs:462-476): h[i] += v, h[sigma^-1(i)] -= v."""
        h = {}
        for i, v in entries:
            h[i] = (h.get(i, 0) + v) % R
            j = sigma(self.n, i)
            h[j] = (h.get(j, 0) - v) % R
        return sorted((i, v) for i, v in h.items() if v)

    def gather(self, family, entries):
        """gather_msm_batch over a base family (kzg.rs:52-67), bases route."""
        if not entries:
            return G1_ZERO
        bases = self.B[family]
        pts = b"".join(bases[i] for i, _ in entries)
        return O.msm_g1(pts, frs(v for _, v in entries), threads=self.threads)

    def commit(self, coeffs):
        """KzgParams::commit over the tau_x powers (kzg.rs:130-146)."""
        if not coeffs:
            return G1_ZERO
        return O.msm_g1(self.kzg_g1[:64 * len(coeffs)], frs(coeffs), threads=self.threads)

    def commit_g2(self, coeffs):
        if not coeffs:
            return G2_ZERO
        return O.msm_g2(self.kzg_g2[:128 * len(coeffs)], frs(coeffs), threads=self.threads)

    # ------------------------------------------------------------ anchor proof
    def prove_anchor(self, w):
        """prove_anchor_traced (dynaverse.rs:149-248) -> anchor proof fields."""
        return self._anchor_bases(w) if self.route == "bases" else self._anchor_scalar(w)

    def _anchor_scalar(self, w):
        n = self.n
        six = 6 * n
        nz = [(i, v) for i, v in enumerate(w) if v]
        h = self.h_sparse(nz)
        dot = lambda col, ent: sum(v * col[i] for i, v in ent) % R
        s = {}
        s["w"] = dot(self.lx, nz)
        s["h"] = dot(self.ly, h)
        dyn = [dot(self.alpha, nz), dot(self.beta, nz), dot(self.hb, nz), dot(self.zb, nz), dot(self.bb, nz)]
        wires = [sum(w[t * n + j] * self.lsx[j] for j in range(n)) % R for t in range(6)]
        cons = []
        adeg = dot(self.adeg, nz)
        for t in range(6):
            sl = [(j, w[t * n + j]) for j in range(n) if w[t * n + j]]
            cons += [dot(self.qac[t], nz), dot(self.qcd, sl), dot(self.qbd, sl), dot(self.dd, sl), adeg,
                     dot(self.bdeg, sl), dot(self.ddeg, sl)]
        pzq = dot(self.pq, nz)
        mq = (wires[3] * wires[4] - wires[5]) * inv(self.zn) % R
        g = g1_of(wires + [s["w"], s["h"]] + dyn + [s["w"], s["h"]] + cons + [pzq, mq])
        s5g2 = g2_of([wires[4]])[0]
        # dynamo: alpha, beta, h, z, b, q (identity), instance_z, instance_h
        a = AnchorFields()
        a.wires = g[:6]
        a.s5_g2 = s5g2
        a.w_commitment, a.h_commitment = g[6], g[7]
        a.dynamo = g[8:13] + [G1_ZERO] + g[13:15]
        a.consistency = g[15:57]
        a.public_zero_quotient, a.multiplication_quotient = g[57], g[58]
        return a

    def _anchor_bases(self, w):
        n, m = self.n, self.m
        padded = list(w) + [0] * (m - len(w))
        w_coeffs = ints(O.ntt(frs(padded), "inverse"))
        w_commitment = self.commit(w_coeffs)
        nz = [(i, v) for i, v in enumerate(padded) if v]
        h = self.h_sparse(nz)
        dyn = self._dynamo(nz, h)
        if dyn[6] != w_commitment:
            raise AssertionError("shared X commitment mismatch")
        wire_coeffs = [ints(O.ntt(frs(padded[t * n:(t + 1) * n]), "inverse")) for t in range(6)]
        a = AnchorFields()
        a.wires = [self.commit(c) for c in wire_coeffs]
        a.s5_g2 = self.commit_g2(wire_coeffs[4])
        a.w_commitment, a.h_commitment = w_commitment, dyn[7]
        a.dynamo = dyn
        cons = []
        full = padded[:6 * n]  # zero from 6n on
        dense = lambda fam, vec: O.msm_g1(b"".join(self.B[fam][:len(vec)]), frs(vec), threads=self.threads)
        adeg = dense("adeg", full)
        for t in range(6):
            sl = padded[t * n:(t + 1) * n]
            cons += [dense(f"qac{t}", full), dense("qcd", sl), dense("qbd", sl), dense("d", sl),
                     adeg, dense("bdeg", sl), dense("ddeg", sl)]
        a.consistency = cons
        # public quotient: w / I_x exactly (PreparedExactDivision, domain.rs:268-300),
        # I_x by a balanced product tree (vanishing_polynomial_balanced, domain.rs:60-75)
        ix = _product_tree([pow(self.wm, i, R) for i in range(6 * n, m)])
        qx = ints(O.poly_div_exact(frs(w_coeffs), frs(ix)))
        a.public_zero_quotient = self.commit(qx)
        prod = ints(O.poly_mul(frs(wire_coeffs[3]), frs(wire_coeffs[4])))
        num = _psub(prod, wire_coeffs[5])
        zn = [R - 1] + [0] * (n - 1) + [1]
        quotient = ints(O.poly_div_exact(frs(num), frs(zn)))
        a.multiplication_quotient = self.commit(quotient)
        return a

    def _dynamo(self, z_entries, h_entries):
        """dynamo_prove_unmasked (dynamo.rs:260-276): five sparse commitments
        over the same entries, q = identity, instance_z over lx, instance_h
        over ly; returned in DynamoProof field order."""
        c = [self.gather(f, z_entries) for f in ("alpha", "beta", "h", "z", "b")]
        return c + [G1_ZERO, self.gather("lx", z_entries), self.gather("ly", h_entries)]

    # ------------------------------------------------------------ opening cache
    def opening_cache(self, w):
        """precompute_anchor_openings (dynaverse.rs:300-311): single-point
        openings q_t[i] = [(s_t - s_t(x_i)) / (X - x_i)] of the three
        multiplication wires at every small-domain point.  Bases route: the
        dense quotient of each opening (kzg.rs:277-295 computes the same
        points through a group FFT); scalar route: (s_t(tau) - v_i)/(tau - x_i)."""
        n = self.n
        cache = []
        for t in range(3, 6):
            vals = w[t * n:(t + 1) * n]
            if self.route == "bases":
                col = self._single_openings(ints(O.ntt(frs(vals), "inverse")))
            else:
                st = sum(v * l for v, l in zip(vals, self.lsx)) % R
                invs = batch_inv([(self.tx - x) % R for x in self.small_points])
                col = g1_of([(st - vals[i]) * invs[i] for i in range(n)])
            cache.append(col)
        return cache

    def _single_openings(self, coeffs):
        """KzgParams::precompute_single_openings (kzg.rs:207-246): the
        Toeplitz product H_j = sum_(l > j) f_l [tau^(l-1-j)] as a circular
        convolution (scalar FFT of the reversed coefficients times the group
        FFT of the powers, one group IFFT), then a group FFT of H over the
        n-point domain gives every opening [(f - f(x_i)) / (X - x_i)]."""
        n = self.n
        degree = len(coeffs) - 1
        if degree == 0:
            return [G1_ZERO] * n
        conv = 1
        while conv < 2 * degree - 1:
            conv <<= 1
        rev = list(reversed(coeffs[1:])) + [0] * (conv - degree)
        scalar_fft = O.ntt(frs(rev), "forward")
        if self._prepared is None or self._prepared[0] != degree:
            powers = self.kzg_g1[:64 * degree] + G1_ZERO * (conv - degree)
            self._prepared = (degree, O.g1_fft(powers, conv, False, threads=self.threads))
        prod = O.g1_scale(self._prepared[1], scalar_fft, threads=self.threads)
        h = O.g1_fft(prod, conv, True, threads=self.threads)
        hs = _split(h[:64 * degree], 64)[::-1] + [G1_ZERO] * (n - degree)
        return _split(O.g1_fft(b"".join(hs), n, False, threads=self.threads), 64)

    # ------------------------------------------------------------ sparse delta proof
    def prove_delta(self, anchor_w, entries, anchor_wires, cache):
        """prove_delta_sparse_traced (dynaverse/sparse.rs:79-276); entries:
        sorted (index, anchor difference) pairs, all nonzero, index < 6n."""
        if self.route == "bases":
            return self._delta_bases(anchor_w, entries, anchor_wires, cache)
        return self._delta_scalar(anchor_w, entries, anchor_wires)

    def _geometry(self, entries):
        n = self.n
        slices = [[] for _ in range(6)]
        affected = set()
        for i, v in entries:
            slices[i // n].append((i % n, v))
            if i >= 3 * n:
                affected.add(i % n)
        return slices, sorted(affected)

    def _delta_bases(self, anchor_w, entries, anchor_wires, cache):
        n = self.n
        d = DeltaFields()
        h = self.h_sparse(entries)
        d.dynamo = self._dynamo(entries, h)
        slices, affected = self._geometry(entries)
        d.changed_wires = [self.gather("lag", sl) for sl in slices]
        cons = []
        for t in range(6):
            s = slices[t]
            cons += [self.gather(f"qac{t}", entries), self.gather("qcd", s), self.gather("qbd", s),
                     self.gather("d", s), self.gather("adeg", entries), self.gather("bdeg", s),
                     self.gather("ddeg", s)]
        d.consistency = cons
        d.public_zero_quotient = self.gather("pq", entries)
        d.changed_w, d.changed_h = d.dynamo[6], d.dynamo[7]
        pts = [self.small_points[i] for i in affected]
        if pts:
            tree = O.Tree(frs(pts))
            weights = ints(tree.inverse_derivatives())
            ai = ints(tree.vanishing())
        else:
            tree, weights, ai = None, [], [1]
        d.affected_g1 = self.commit(ai)
        d.affected_g2 = self.commit_g2(ai)
        inverses = batch_inv(pts) if pts else []
        b_entries = [(i, n * inverses[j] % R * weights[j] % R) for j, i in enumerate(affected)]
        if not affected:
            d.unaffected_g1, d.unaffected_g2 = self.multiplication_vanishing_g1, self.multiplication_divisor
        else:
            d.unaffected_g1 = self.gather("lag", b_entries)
            d.unaffected_g2 = O.msm_g2(b"".join(self.lag_g2[i] for i in affected), frs(v for _, v in b_entries),
                                       threads=self.threads)
        interp = lambda vals: ints(tree.interpolate(frs(vals))) if pts else [0]
        cauchy = lambda vals: ints(tree.cauchy_sums(frs(vals))) if pts else []
        cw = cauchy(weights)
        inv_n = inv(n)
        anchor_local, changed_local, zero_q, changed_open = [], [], [], []
        for t in range(3):
            sl = dict(slices[t + 3])
            av = [anchor_w[(t + 3) * n + i] for i in affected]
            vals = [sl.get(i, 0) for i in affected]
            anchor_local.append(interp(av))
            changed_local.append(interp(vals))
            cv = cauchy([v * x % R for v, x in zip(vals, pts)])
            lag = [(i, (vals[j] * cw[j] + weights[j] * inverses[j] % R * cv[j]) % R) for j, i in enumerate(affected)]
            opn = [(i, vals[j] * weights[j] % R) for j, i in enumerate(affected)]
            changed_open.append(g1_add(self.gather("lag", lag), self.gather("open_u", opn)))
            zero_q.append(interp([vals[j] * inv(weights[j]) % R * pts[j] % R * inv_n % R
                                  for j in range(len(affected))]))
        updated = [_padd(anchor_local[t], changed_local[t]) for t in range(3)]
        prod = ints(O.poly_mul(frs(updated[0]), frs(updated[1])))
        num = _psub(prod, updated[2])
        local_q = ints(O.poly_div_exact(frs(num), frs(ai)))
        if not affected:
            d.anchor_openings = list(anchor_wires[3:6])
        else:
            sel = list(zip(affected, weights))
            d.anchor_openings = [O.msm_g1(b"".join(cache[t][i] for i, _ in sel), frs(v for _, v in sel),
                                          threads=self.threads) for t in range(3)]
        d.anchor_local = [self.commit(c) for c in anchor_local]
        d.changed_local = [self.commit(c) for c in changed_local]
        d.unaffected_zero = [self.commit(c) for c in zero_q]
        d.local_quotient = self.commit(local_q)
        d.updated_s5_g2 = self.commit_g2(updated[1])
        d.changed_openings = changed_open
        if tree is not None:
            tree.close()
        return d

    def _delta_scalar(self, anchor_w, entries, anchor_wires):
        """Every field of the sparse delta proof as a scalar at tau_x: the
        sparse sums of the linear part, and the polynomials of the affected
        set through their values at tau_x (A, the interpolants r, r*, the
        dense quotients (s - r)/A, (delta - r*)/A, delta A/(X^n - 1) and
        (u0 u1 - u2)/A that the sparse steps reproduce)."""
        n = self.n
        tx = self.tx
        h = self.h_sparse(entries)
        dot = lambda col, ent: sum(v * col[i] for i, v in ent) % R
        slices, affected = self._geometry(entries)
        lin = [dot(self.alpha, entries), dot(self.beta, entries), dot(self.hb, entries), dot(self.zb, entries),
               dot(self.bb, entries), dot(self.lx, entries), dot(self.ly, h)]
        wires = [dot(self.lsx, sl) for sl in slices]
        cons = []
        adeg = dot(self.adeg, entries)
        for t in range(6):
            s = slices[t]
            cons += [dot(self.qac[t], entries), dot(self.qcd, s), dot(self.qbd, s), dot(self.dd, s), adeg,
                     dot(self.bdeg, s), dot(self.ddeg, s)]
        pzq = dot(self.pq, entries)
        pts = [self.small_points[i] for i in affected]
        a_tau = 1
        for x in pts:
            a_tau = a_tau * (tx - x) % R
        # A'(x_k) = prod_{j != k} (x_k - x_j)
        deriv = []
        for k, xk in enumerate(pts):
            p = 1
            for j, xj in enumerate(pts):
                if j != k:
                    p = p * (xk - xj) % R
            deriv.append(p)
        weights = batch_inv(deriv) if pts else []
        lag_tau = [self.lsx[i] for i in affected]
        inv_tx = batch_inv([(tx - x) % R for x in pts]) if pts else []

        def interp_tau(vals):  # sum v_k w_k A(tau)/(tau - x_k)
            return sum(v * wk % R * inv_t for v, wk, inv_t in zip(vals, weights, inv_tx)) % R * a_tau % R

        unaffected = (self.zn * inv(a_tau)) % R
        a_inv = inv(a_tau)
        r, rs, zq, ao, co = [], [], [], [], []
        for t in range(3):
            sl = dict(slices[t + 3])
            av = [anchor_w[(t + 3) * n + i] for i in affected]
            vals = [sl.get(i, 0) for i in affected]
            rt, rst = interp_tau(av), interp_tau(vals)
            r.append(rt)
            rs.append(rst)
            st = sum(anchor_w[(t + 3) * n + j] * self.lsx[j] for j in range(n)) % R
            dt = sum(v * l for v, l in zip(vals, lag_tau)) % R  # the slice's delta polynomial at tau
            ao.append((st - rt) * a_inv % R)
            co.append((dt - rst) * a_inv % R)
            zq.append(dt * inv(unaffected) % R)  # delta / B with B(tau) = (tau^n - 1) / A(tau)
        u = [(r[t] + rs[t]) % R for t in range(3)]
        lq = (u[0] * u[1] - u[2]) * a_inv % R
        g = g1_of(wires + lin[:5] + lin[5:7] + cons + [pzq, a_tau, unaffected] + r + rs + co + zq + [lq] +
                  (ao if affected else []))
        gg = g2_of([a_tau, unaffected, u[1]])
        d = DeltaFields()
        d.changed_wires = g[:6]
        d.dynamo = g[6:11] + [G1_ZERO] + g[11:13]
        d.changed_w, d.changed_h = g[11], g[12]
        d.consistency = g[13:55]
        d.public_zero_quotient = g[55]
        d.affected_g1, d.unaffected_g1 = g[56], g[57]
        d.affected_g2, d.unaffected_g2 = gg[0], gg[1]
        d.anchor_local = g[58:61]
        d.changed_local = g[61:64]
        d.changed_openings = g[64:67]
        d.unaffected_zero = g[67:70]
        d.local_quotient = g[70]
        d.anchor_openings = g[71:74] if affected else list(anchor_wires[3:6])
        d.updated_s5_g2 = gg[2]
        return d

    # ------------------------------------------------------------ verifier
    def equations(self, pub, proof):
        """The pairing-product equations and group checks of verify_traced
        (dynaverse.rs:978-1119) for a proof object.  Returns (terms, groups):
        terms is a list of equations, each a list of (G1, G2) pairs whose
        pairing product must be one (right-hand sides negated as
        product_equal does, verification.rs:80-92); groups is the list of
        G1 identities that must hold."""
        g1, g2 = self.g1, self.g2
        eqs, groups = [], []

        def eq(left, rights):
            eqs.append([left] + [(g1_neg(p), q) for p, q in rights])

        def dynamo(dp, w_c, h_c):
            groups.append(w_c == dp[6] and h_c == dp[7])
            alpha, beta, hh, z, b, q, iz, ih = dp
            eq((iz, self.vk_u), [(alpha, self.vk_xm1), (beta, self.vk_x), (ih, self.vk_inv_m), (q, self.vk_ym1)])
            eq((iz, self.vk_ym), [(z, g2)])
            eq((ih, self.vk_xm), [(hh, g2)])
            eq((beta, self.vk_x2), [(b, g2)])

        def consistency(a, wires, cons):
            for t in range(6):
                qac, qcd, qbd, d, adeg, bdeg, ddeg = cons[7 * t:7 * t + 7]
                b = wires[t]
                eq((g1_sub(a, d), g2), [(qac, self.vk_z_in[t]), (qcd, self.vk_x_minus_y)])
                eq((g1_sub(b, d), g2), [(qbd, self.vk_x_minus_ly)])
                eq((a, self.vk_ym), [(adeg, g2)])
                eq((b, self.vk_ym), [(bdeg, g2)])
                eq((d, self.vk_xm), [(ddeg, g2)])

        an = proof.anchor
        dynamo(an.dynamo, an.w_commitment, an.h_commitment)
        consistency(an.w_commitment, an.wires, an.consistency)
        eq((an.public_zero_quotient, self.public_zero_divisor), [(an.w_commitment, g2)])
        groups.append(g1_add(an.wires[0], an.wires[1]) == an.wires[2])
        eq((an.wires[4], g2), [(g1, an.s5_g2)])
        eq((an.wires[3], an.s5_g2), [(an.wires[5], g2), (an.multiplication_quotient, self.multiplication_divisor)])
        dl = proof.delta
        if dl is not None:
            dynamo(dl.dynamo, dl.changed_w, dl.changed_h)
            consistency(dl.changed_w, dl.changed_wires, dl.consistency)
            eq((dl.public_zero_quotient, self.public_zero_divisor), [(dl.changed_w, g2)])
            groups.append(g1_add(dl.changed_wires[0], dl.changed_wires[1]) == dl.changed_wires[2])
            eq((dl.affected_g1, g2), [(g1, dl.affected_g2)])
            eq((dl.unaffected_g1, g2), [(g1, dl.unaffected_g2)])
            eq((dl.affected_g1, dl.unaffected_g2), [(self.multiplication_vanishing_g1, g2)])
            ru = [g1_add(dl.anchor_local[i], dl.changed_local[i]) for i in range(3)]
            eq((ru[1], g2), [(g1, dl.updated_s5_g2)])
            eq((ru[0], dl.updated_s5_g2), [(ru[2], g2), (dl.local_quotient, dl.affected_g2)])
            for i in range(3):
                eq((dl.anchor_openings[i], dl.affected_g2), [(g1_sub(an.wires[3 + i], dl.anchor_local[i]), g2)])
                eq((dl.changed_openings[i], dl.affected_g2),
                   [(g1_sub(dl.changed_wires[3 + i], dl.changed_local[i]), g2)])
                eq((dl.unaffected_zero[i], dl.unaffected_g2), [(dl.changed_wires[3 + i], g2)])
        # public inputs: anchor h + delta h + [public]_h == 0
        pub_nz = [(k, v) for k, v in enumerate(pub) if v]
        public_h = O.msm_g1(b"".join(self.public_h_bases[k] for k, _ in pub_nz), frs(v for _, v in pub_nz)) \
            if pub_nz else G1_ZERO
        total = g1_add(an.h_commitment, dl.changed_h if dl is not None else G1_ZERO)
        groups.append(g1_add(total, public_h) == G1_ZERO)
        return eqs, groups

    def verify(self, pub, proof, threads=0):
        """verify_traced in Product mode (dynaverse.rs:978-1016): every
        equation and group identity must hold."""
        if len(pub) != self.n or proof.anchor_generation > proof.generation or \
                (proof.delta is not None) != (proof.anchor_generation < proof.generation):
            return False
        eqs, groups = self.equations(pub, proof)
        g1 = b"".join(p for e in eqs for p, _ in e)
        g2 = b"".join(q for e in eqs for _, q in e)
        offs = [0]
        for e in eqs:
            offs.append(offs[-1] + len(e))
        try:
            return all(groups) and all(O.pairing_check(g1, g2, offs, threads=threads))
        except ValueError:  # a point off its curve never deserialises (codec.rs:25-111)
            return False


# ------------------------------------------------------------------ proof objects
class AnchorFields:
    wires = s5_g2 = w_commitment = h_commitment = dynamo = consistency = None
    public_zero_quotient = multiplication_quotient = None

    def to_bytes(self) -> bytes:
        out = b"".join(self.wires) + self.s5_g2 + self.w_commitment + self.h_commitment + \
            b"".join(self.dynamo) + b"".join(self.consistency) + self.public_zero_quotient + \
            self.multiplication_quotient
        assert len(out) == ANCHOR_BYTES
        return out


class DeltaFields:
    changed_wires = changed_w = changed_h = dynamo = consistency = public_zero_quotient = None
    affected_g1 = affected_g2 = unaffected_g1 = unaffected_g2 = None
    anchor_local = changed_local = updated_s5_g2 = anchor_openings = changed_openings = None
    unaffected_zero = local_quotient = None

    def to_bytes(self) -> bytes:
        out = b"".join(self.changed_wires) + self.changed_w + self.changed_h + b"".join(self.dynamo) + \
            b"".join(self.consistency) + self.public_zero_quotient + self.affected_g1 + self.affected_g2 + \
            self.unaffected_g1 + self.unaffected_g2 + b"".join(self.anchor_local) + \
            b"".join(self.changed_local) + self.updated_s5_g2 + b"".join(self.anchor_openings) + \
            b"".join(self.changed_openings) + b"".join(self.unaffected_zero) + self.local_quotient
        assert len(out) == DELTA_BYTES
        return out


class Proof:
    def __init__(self, anchor, delta, anchor_generation, generation):
        self.anchor, self.delta = anchor, delta
        self.anchor_generation, self.generation = anchor_generation, generation

    def to_bytes(self) -> bytes:
        d = self.delta.to_bytes() if self.delta is not None else bytes(DELTA_BYTES)
        return self.anchor.to_bytes() + d + \
            struct.pack("<QQQ", 1 if self.delta is not None else 0, self.anchor_generation, self.generation)


def parse_proof(b: bytes) -> Proof:
    """Proof bytes -> fields (the inverse of Proof.to_bytes)."""
    assert len(b) == PROOF_BYTES
    pos = [0]

    def take(k):
        v = b[pos[0]:pos[0] + k]
        pos[0] += k
        return v
    g = lambda: take(64)
    a = AnchorFields()
    a.wires = [g() for _ in range(6)]
    a.s5_g2 = take(128)
    a.w_commitment, a.h_commitment = g(), g()
    a.dynamo = [g() for _ in range(8)]
    a.consistency = [g() for _ in range(42)]
    a.public_zero_quotient, a.multiplication_quotient = g(), g()
    d = DeltaFields()
    d.changed_wires = [g() for _ in range(6)]
    d.changed_w, d.changed_h = g(), g()
    d.dynamo = [g() for _ in range(8)]
    d.consistency = [g() for _ in range(42)]
    d.public_zero_quotient, d.affected_g1 = g(), g()
    d.affected_g2 = take(128)
    d.unaffected_g1 = g()
    d.unaffected_g2 = take(128)
    d.anchor_local = [g() for _ in range(3)]
    d.changed_local = [g() for _ in range(3)]
    d.updated_s5_g2 = take(128)
    d.anchor_openings = [g() for _ in range(3)]
    d.changed_openings = [g() for _ in range(3)]
    d.unaffected_zero = [g() for _ in range(3)]
    d.local_quotient = g()
    has, ag, gen = struct.unpack("<QQQ", take(24))
    return Proof(a, d if has else None, ag, gen)


# ------------------------------------------------------------------ session
class Session:
    """UpdateSession (dynaverse/session.rs:10-142) over Params.  With
    scalar_anchors, anchors and opening caches (session start and
    re-anchors) come from the scalar route even on the bases route, whose
    sparse proofs and verifier then run on them: the values are identical
    (tests/test_oracle_dynaverse.py), and the CPU baseline times the sparse
    path without minutes of dense setup per anchor."""

    def __init__(self, params: Params, pub, witness, verify=True, scalar_anchors=False):
        p = self.p = params
        n = p.n
        if len(pub) != n or len(witness) != 6 * n:
            raise ValueError("instance or witness length differs from circuit")
        check_gates(n, pub, witness, range(n))
        self.scalar_anchors = scalar_anchors
        self.pub = list(pub)
        self.anchor = list(witness)
        self.current = list(witness)
        a, self.cache = self._anchor(witness)
        self.proof = Proof(a, None, 0, 0)
        if verify and not p.verify(self.pub, self.proof):
            raise AssertionError("initial session proof failed verification")
        self.delta = {}
        self.last_rebuilt = False

    def _anchor(self, w):
        p = self.p
        if self.scalar_anchors and p.route == "bases":
            p.route = "scalar"
            try:
                return p.prove_anchor(w), p.opening_cache(w)
            finally:
                p.route = "bases"
        return p.prove_anchor(w), (p.opening_cache(w) if p.route == "bases" else None)

    def anchor_distance(self):
        return len(self.delta)

    def update(self, indices, values, pub_indices=(), pub_values=(), verify=True):
        """UpdateSession::update_with_public_inputs; returns the new proof
        (the current one for a no-op) or raises ValueError and leaves the
        session unchanged."""
        p = self.p
        n = p.n
        edits = canonicalize(list(indices), list(values), 6 * n)
        pedits = canonicalize(list(pub_indices), list(pub_values), n)
        dirty, changed = set(), False
        for i, v in edits.items():
            if v != self.current[i]:
                changed = True
                dirty.add(i % n)
        for i, v in pedits.items():
            if v != self.pub[i]:
                changed = True
                dirty.add(i)
        if not changed:
            return self.proof
        w = list(self.current)
        for i, v in edits.items():
            w[i] = v
        pub = list(self.pub)
        for i, v in pedits.items():
            pub[i] = v
        check_gates(n, pub, w, sorted(dirty))
        generation = self.proof.generation + 1
        delta = dict(self.delta)
        for i, v in edits.items():
            diff = (v - self.anchor[i]) % R
            if diff == 0:
                delta.pop(i, None)
            else:
                delta[i] = diff
        if len(delta) >= p.rebuild_interval:
            # update_proof_backend's rebuild branch (dynaverse.rs:423-437)
            check_gates(n, pub, w, range(n))
            a, cache = self._anchor(w)
            proof = Proof(a, None, generation, generation)
            if verify and not p.verify(pub, proof):
                raise ValueError("updated proof failed public verification")
            self.anchor = list(w)
            self.cache = cache
            self.delta = {}
            self.last_rebuilt = True
        else:
            entries = sorted(delta.items())
            d = p.prove_delta(self.anchor, entries, self.proof.anchor.wires, self.cache)
            proof = Proof(self.proof.anchor, d, self.proof.anchor_generation, generation)
            if verify and not p.verify(pub, proof):
                raise ValueError("sparse session proof failed verification")
            self.delta = delta
            self.last_rebuilt = False
        self.current, self.pub, self.proof = w, pub, proof
        return proof


# ------------------------------------------------------------------ small polynomial helpers
def _split(b: bytes, size: int):
    return [b[i:i + size] for i in range(0, len(b), size)]


def _product_tree(roots):
    """prod (X - r) by pairwise products (the oracle's FFT poly_mul)."""
    if not roots:
        return [1]
    level = [[(-r) % R, 1] for r in roots]
    while len(level) > 1:
        nxt = []
        for i in range(0, len(level) - 1, 2):
            nxt.append(ints(O.poly_mul(frs(level[i]), frs(level[i + 1]))))
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    return level[0]


def _pmul(a, b):
    out = [0] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            out[i + j] = (out[i + j] + x * y) % R
    return out


def _trim(a):
    a = list(a)
    while len(a) > 1 and a[-1] == 0:
        a.pop()
    return a or [0]


def _padd(a, b):
    out = [0] * max(len(a), len(b), 1)
    for i, v in enumerate(a):
        out[i] = (out[i] + v) % R
    for i, v in enumerate(b):
        out[i] = (out[i] + v) % R
    return out


def _psub(a, b):
    out = [0] * max(len(a), len(b), 1)
    for i, v in enumerate(a):
        out[i] = (out[i] + v) % R
    for i, v in enumerate(b):
        out[i] = (out[i] - v) % R
    return _trim(out)
