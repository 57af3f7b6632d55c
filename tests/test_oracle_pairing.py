"""Pins the oracle's pairing (the optimal ate pairing of
crates/protocol/src/verification.rs:37-144) to tests/golden/pairing.json,
made by tests/golden/make_pairing_golden.py from a pure-Python flat-Fq12
pairing that shares no code with it, and checks the constants that the
CUDA pairing embeds.  No GPU."""
import json
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import bn254_py as b  # noqa: E402


@pytest.fixture(scope="module")
def pairing_golden():
    with open(os.path.join(ROOT, "tests", "golden", "pairing.json")) as f:
        return json.load(f)


def test_hard_part_digits_and_python_pairing_properties():
    z, q, r = b.BN_SEED, b.Q, b.R
    digits = [12 * z**3 + 12 * z**2 + 6 * z + 1, 12 * z**3 + 6 * z**2 + 4 * z,
              12 * z**3 + 6 * z**2 + 6 * z, 12 * z**3 + 6 * z**2 + 4 * z - 1]
    assert (q**4 - q**2 + 1) % r == 0
    assert sum(d * q**i for i, d in enumerate(digits)) == b.FINAL_EXP_MULTIPLE * (q**4 - q**2 + 1) // r
    assert b.FINAL_EXP_MULTIPLE % r != 0  # verdicts equal the plain reduced pairing's
    e = b.pairing(b.G1_GEN, b.G2_GEN)
    assert e != b.F12_ONE and b.f12pow(e, r) == b.F12_ONE
    assert b.pairing(b.g1_mul(b.G1_GEN, 3), b.g2_mul(b.G2_GEN, 5)) == b.f12pow(e, 15)


def test_oracle_matches_golden_pairings(oracle, pairing_golden):
    for case in pairing_golden["single"]:
        assert oracle.pairing(bytes.fromhex(case["g1"]), bytes.fromhex(case["g2"])).hex() == case["gt"]


def test_oracle_matches_golden_equations(oracle, pairing_golden):
    g1 = b"".join(bytes.fromhex(x) for e in pairing_golden["equations"] for x in e["g1"])
    g2 = b"".join(bytes.fromhex(x) for e in pairing_golden["equations"] for x in e["g2"])
    offsets = [0]
    for e in pairing_golden["equations"]:
        offsets.append(offsets[-1] + len(e["g1"]))
    assert oracle.pairing_check(g1, g2, offsets) == [e["holds"] for e in pairing_golden["equations"]]


def test_oracle_rejects_off_curve_points(oracle):
    bad = (1).to_bytes(32, "little") + (1).to_bytes(32, "little")
    with pytest.raises(ValueError):
        oracle.pairing(bad, b.g2_bytes(b.G2_GEN))


def _c_words(text, name):
    m = re.search(name + r"[^=]*=\s*\{(.*?)\};", text, flags=re.S)
    return [int(x, 16) for x in re.findall(r"0x[0-9a-fA-F]+", m.group(1))]


def test_device_pairing_constants():
    src = open(os.path.join(ROOT, "zkp-dynaverse_b200", "csrc", "pairing.cu")).read()
    q = b.Q
    mont = lambda v: (v << 256) % q
    words = lambda ws: sum(w << (32 * i) for i, w in enumerate(ws))
    g = b.f2pow((9, 1), (q - 1) // 6)
    f1 = _c_words(src, "FROB1")
    f2 = _c_words(src, "FROB2")
    for j in range(6):
        gj = b.f2pow(g, j)
        assert words(f1[16 * j:16 * j + 8]) == mont(gj[0]) and words(f1[16 * j + 8:16 * j + 16]) == mont(gj[1])
        assert words(f2[8 * j:8 * j + 8]) == mont((gj[0] ** 2 + gj[1] ** 2) % q)
    m = re.search(r"NAF_6Z2\[(\d+)\]\s*=\s*\{([^}]*)\}", src)
    assert [int(x) for x in m.group(2).split(",")] == b.naf(6 * b.BN_SEED + 2)
    naf = b.naf(6 * b.BN_SEED + 2)
    lines = (len(naf) - 1) + sum(1 for d in naf[1:] if d) + 2  # doublings, additions, two Frobenius lines
    assert int(re.search(r"constexpr int LINES = (\d+);", src).group(1)) == lines
    m = re.search(r"WNAF_Z\[(\d+)\]\s*=\s*\{([^}]*)\}", src)
    digits = [int(x) for x in m.group(2).split(",")]
    assert len(digits) == int(m.group(1)) == int(re.search(r"WNAF_Z_LEN = (\d+);", src).group(1))
    assert digits == _wnaf(b.BN_SEED, 4)
    value = 0
    for d in digits:
        value = 2 * value + d
    assert value == b.BN_SEED and digits[0] > 0
    assert sum(1 for d in digits if d) == 14


def _wnaf(k, w):
    """Width-w NAF of k, most significant digit first: odd digits in
    (-2^(w-1), 2^(w-1)), any two nonzero digits at least w places apart."""
    out = []
    while k:
        d = 0
        if k & 1:
            d = k % (1 << w)
            if d >= 1 << (w - 1):
                d -= 1 << w
            k -= d
        out.append(d)
        k >>= 1
    return out[::-1]


def test_divstep_inverse_constants():
    """R^3 mod p (R = 2^256) of both fields, the constant that turns the
    divstep inverse of a Montgomery value back into Montgomery form."""
    src = open(os.path.join(ROOT, "zkp-dynaverse_b200", "csrc", "field.cuh")).read()
    fr = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
    for cfg, mod in (("FqCfg", b.Q), ("FrCfg", fr)):
        body = src[src.index("struct " + cfg):]
        body = body[:body.index("};")]
        words = [int(re.search(r"R3%d = 0x([0-9a-f]+)u" % i, body).group(1), 16) for i in range(8)]
        assert sum(w << (32 * i) for i, w in enumerate(words)) == pow(1 << 256, 3, mod)
        inv = int(re.search(r"INV = 0x([0-9a-f]+)u", body).group(1), 16)
        assert (inv * mod) % (1 << 32) == (1 << 32) - 1  # -p^-1 mod 2^32, whose negation mod 2^30 is p^-1
