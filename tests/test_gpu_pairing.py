"""Device pairing checks (dvgpu_bn254_pairing_check / dvgpu_bn254_pairing)
against the golden pairings of tests/golden/pairing.json and the oracle, on
the equation shapes of crates/protocol/src/verification.rs:37-144 (a left
pair and negated right pairs, one final exponentiation per equation)."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001


@pytest.fixture(scope="module")
def pairing_golden():
    with open(os.path.join(ROOT, "tests", "golden", "pairing.json")) as f:
        return json.load(f)


def test_pairings_match_golden(backend, pairing_golden):
    g1 = b"".join(bytes.fromhex(c["g1"]) for c in pairing_golden["single"])
    g2 = b"".join(bytes.fromhex(c["g2"]) for c in pairing_golden["single"])
    got = backend.pairing(g1, g2)
    for i, c in enumerate(pairing_golden["single"]):
        assert got[384 * i:384 * (i + 1)].hex() == c["gt"], f"pair {i}"


def test_equations_match_golden(backend, pairing_golden):
    eqs = pairing_golden["equations"]
    g1 = b"".join(bytes.fromhex(x) for e in eqs for x in e["g1"])
    g2 = b"".join(bytes.fromhex(x) for e in eqs for x in e["g2"])
    offsets = [0]
    for e in eqs:
        offsets.append(offsets[-1] + len(e["g1"]))
    assert backend.pairing_check(g1, g2, offsets) == [e["holds"] for e in eqs]


def _neg_g1(p):
    if not any(p):
        return p
    y = int.from_bytes(p[32:], "little")
    q = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
    return p[:32] + ((q - y) % q).to_bytes(32, "little")


def test_random_batches_match_oracle(backend, oracle):
    """Equations e(a P, c Q) = e(ac P, Q) (and broken ones), 1..4 terms,
    empty equations and infinity terms, against the oracle's verdicts; single
    pairings against the oracle's GT bytes."""
    n = 96
    sa = oracle.uniform_fr(5001, n)
    sc = oracle.uniform_fr(5002, n)
    ints = lambda buf: [int.from_bytes(buf[32 * i:32 * i + 32], "little") for i in range(len(buf) // 32)]
    a, c = ints(sa), ints(sc)
    ac = b"".join(((x * y + (k % 3 == 1)) % R_MOD).to_bytes(32, "little") for k, (x, y) in enumerate(zip(a, c)))
    pa = oracle.fixed_base_g1(sa)
    pac = oracle.fixed_base_g1(ac)
    qc = oracle.fixed_base_g2(sc)
    one = (1).to_bytes(32, "little")
    gen1 = oracle.fixed_base_g1(one)
    gen2 = oracle.fixed_base_g2(one)
    g1, g2, offsets = [], [], [0]
    for k in range(n):
        terms = [(pa[64 * k:64 * k + 64], qc[128 * k:128 * k + 128]),
                 (_neg_g1(pac[64 * k:64 * k + 64]), gen2)]
        if k % 5 == 2:
            terms.append((bytes(64), gen2))           # infinity contributes one
        if k % 7 == 3:
            terms.append((gen1, bytes(128)))
        if k % 11 == 4:
            terms = []                                # empty product holds
        for p, q in terms:
            g1.append(p)
            g2.append(q)
        offsets.append(offsets[-1] + len(terms))
    g1, g2 = b"".join(g1), b"".join(g2)
    got = backend.pairing_check(g1, g2, offsets)
    assert got == oracle.pairing_check(g1, g2, offsets)
    assert sum(got) > 0 and not all(got)
    m = 24
    assert backend.pairing(pa[:64 * m], qc[:128 * m]) == oracle.pairing(pa[:64 * m], qc[:128 * m])
    # one G2 point repeated: prepared once inside the call
    assert backend.pairing(pa[:64 * m], gen2 * m) == oracle.pairing(pa[:64 * m], gen2 * m)


def test_bilinearity_on_device(backend, oracle):
    s = oracle.uniform_fr(5010, 2)
    a, c = (int.from_bytes(s[i:i + 32], "little") for i in (0, 32))
    one = (1).to_bytes(32, "little")
    g1 = oracle.fixed_base_g1(s[:32] + (a * c % R_MOD).to_bytes(32, "little") + one)
    g2 = oracle.fixed_base_g2(s[32:] + one + (a * c % R_MOD).to_bytes(32, "little"))
    e = backend.pairing(g1[:64] + g1[64:128] + g1[128:], g2[:128] + g2[128:256] + g2[256:])
    assert e[:384] == e[384:768] == e[768:]  # e(aP, cQ) = e(acP, Q) = e(P, acQ)


def test_invalid_points_are_rejected(backend, oracle, dv):
    one = (1).to_bytes(32, "little")
    gen1, gen2 = oracle.fixed_base_g1(one), oracle.fixed_base_g2(one)
    off_curve = one + one
    with pytest.raises(dv.DvgpuError) as e:
        backend.pairing_check(gen1 + off_curve, gen2 + gen2, [0, 1, 2])
    assert e.value.status == -1 and "G1" in e.value.message and "1" in e.value.message
    with pytest.raises(dv.DvgpuError) as e:
        backend.pairing(gen1, bytes(64) + one * 2)
    assert e.value.status == -1 and "G2" in e.value.message
    with pytest.raises(dv.DvgpuError):
        backend.pairing_check(gen1, gen2, [1, 1])
    assert backend.pairing_check(gen1, gen2, [0, 0, 1]) == [True, False]


def test_prepared_g2_points_across_calls(backend, oracle, dv):
    """Preparations kept on the device (G2Prepared): the same verdicts as the
    plain check for equations that share prepared points, through two calls,
    plus infinity, empty equations and bad handles or indices."""
    n = 48
    sa, sc = oracle.uniform_fr(5101, n), oracle.uniform_fr(5102, n)
    ints = lambda buf: [int.from_bytes(buf[32 * i:32 * i + 32], "little") for i in range(len(buf) // 32)]
    a, c = ints(sa), ints(sc)
    one = (1).to_bytes(32, "little")
    # prepared points: [c_0]G2 .. [c_3]G2, the generator, infinity
    qs = oracle.fixed_base_g2(sc[:128] + one) + bytes(128)
    h = backend.g2_prepare(qs)
    try:
        g1, qidx, plain_g2, offsets = [], [], [], [0]
        for k in range(n):
            j = k % 4
            x = a[k] * c[j] % R_MOD
            if k % 3 == 1:
                x = (x + 1) % R_MOD
            p1 = oracle.fixed_base_g1(sa[32 * k:32 * k + 32])
            p2 = _neg_g1(oracle.fixed_base_g1(x.to_bytes(32, "little")))
            terms = [(p1, j), (p2, 4)]
            if k % 5 == 0:
                terms.append((p1, 5))  # infinity on the G2 side contributes one
            for p, q in terms:
                g1.append(p)
                qidx.append(q)
                plain_g2.append(qs[128 * q:128 * q + 128])
            offsets.append(offsets[-1] + len(terms))
        offsets.append(offsets[-1])  # an empty equation holds
        g1 = b"".join(g1)
        expect = backend.pairing_check(g1, b"".join(plain_g2), offsets)
        assert expect == oracle.pairing_check(g1, b"".join(plain_g2), offsets)
        assert expect[-1] and sum(expect) == 1 + sum(1 for k in range(n) if k % 3 != 1)
        for _ in range(2):
            assert backend.pairing_check_prepared(g1, h, qidx, offsets) == expect
        with pytest.raises(dv.DvgpuError, match="index out of range"):
            backend.pairing_check_prepared(g1[:64], h, [6], [0, 1])
    finally:
        backend.g2_prepared_release(h)
    with pytest.raises(dv.DvgpuError, match="unknown prepared"):
        backend.pairing_check_prepared(g1[:64], h, [0], [0, 1])
    with pytest.raises(dv.DvgpuError, match="invalid G2 point at index 1"):
        backend.g2_prepare(qs[:128] + one + one + bytes(64))


def test_multi_miller_loop_in_large_batches(backend, oracle):
    """Batches of more prepared terms than one wave of per-term groups run
    one multi-Miller loop per equation: 3100 cache-check equations
    e(L, G) e(-R, D_j) = 1 over three divisors (every third one broken), with
    three-term equations (an infinity term on either side), one-term and
    empty ones; verdicts by construction, through the kept preparations and
    through the plain call, and the oracle on a sample."""
    n = 3100
    sa = oracle.uniform_fr(5201, n)
    sd = oracle.uniform_fr(5202, 3)
    a = [int.from_bytes(sa[32 * i:32 * i + 32], "little") for i in range(n)]
    d = [int.from_bytes(sd[32 * j:32 * j + 32], "little") for j in range(3)]
    one = (1).to_bytes(32, "little")
    qs = oracle.fixed_base_g2(one + sd) + bytes(128)  # G, D_0, D_1, D_2, infinity
    rs = b"".join(((a[i] * pow(d[i % 3], R_MOD - 2, R_MOD) + (i % 3 == 2)) % R_MOD).to_bytes(32, "little")
                  for i in range(n))
    left, right = oracle.fixed_base_g1(sa), oracle.fixed_base_g1(rs)
    g1, qidx, offsets, expect = [], [], [0], []
    for i in range(n):
        lp, rp = left[64 * i:64 * i + 64], _neg_g1(right[64 * i:64 * i + 64])
        terms = [(lp, 0), (rp, 1 + i % 3)]
        if i % 13 == 5:
            terms.append((lp, 4))
        if i % 17 == 6:
            terms.insert(1, (bytes(64), 2))
        if i % 29 == 7:
            terms = [(bytes(64), 0)]
        if i % 31 == 8:
            terms = []
        for p, q in terms:
            g1.append(p)
            qidx.append(q)
        offsets.append(offsets[-1] + len(terms))
        expect.append(len(terms) < 2 or i % 3 != 2)
    assert offsets[-1] > 148 * 8 * 5
    g1 = b"".join(g1)
    g2 = b"".join(qs[128 * q:128 * q + 128] for q in qidx)
    h = backend.g2_prepare(qs)
    try:
        assert backend.pairing_check_prepared(g1, h, qidx, offsets) == expect
    finally:
        backend.g2_prepared_release(h)
    assert backend.pairing_check(g1, g2, offsets) == expect
    m = 64
    sub = offsets[m]
    assert backend.pairing_check(g1[:64 * sub], g2[:128 * sub], offsets[:m + 1]) == \
        oracle.pairing_check(g1[:64 * sub], g2[:128 * sub], offsets[:m + 1])
