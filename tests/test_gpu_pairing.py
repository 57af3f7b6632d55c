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
