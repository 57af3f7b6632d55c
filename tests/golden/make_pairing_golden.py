"""Generate tests/golden/pairing.json from the pure-Python optimal ate pairing
in bn254_py.py (flat Fq12, affine twist arithmetic, plain exponentiation).

Run from the repository root:  python tests/golden/make_pairing_golden.py

Cases: single pairings e(P, Q) of generator multiples with seeded scalars
(and infinity on either side, which gives one), and pairing-product
equations prod e(P_k, Q_k) = 1 in the form the reference's product check
builds them (crates/protocol/src/verification.rs:79-103: the left pair,
then the right pairs with negated G1 points): holding ones, with the
scalar relation broken, and with three terms.
"""
import json
import os
import random
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import bn254_py as b  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pairing.json")


def main():
    rng = random.Random(20261203)
    g1, g2 = b.G1_GEN, b.G2_GEN
    pairs = []
    for k in range(4):
        s, t = rng.randrange(1, b.R), rng.randrange(1, b.R)
        pairs.append((b.g1_mul(g1, s), b.g2_mul(g2, t)))
    pairs = [(g1, g2), (None, g2), (g1, None)] + pairs + [(b.g1_neg(g1), g2)]
    single = [{"g1": b.g1_bytes(p).hex(), "g2": b.g2_bytes(q).hex(), "gt": b.gt_bytes(b.pairing(p, q)).hex()}
              for p, q in pairs]
    eqs = []
    for case in range(6):
        a, c = rng.randrange(1, b.R), rng.randrange(1, b.R)
        # e(aP, cQ) = e(acP, Q): left (aP, cQ), right (acP, Q) -> terms (aP, cQ), (-acP, Q)
        ac = a * c % b.R if case % 2 == 0 else (a * c + 1) % b.R
        terms = [(b.g1_mul(g1, a), b.g2_mul(g2, c)), (b.g1_neg(b.g1_mul(g1, ac)), g2)]
        if case >= 4:  # three terms: e(aP, cQ) = e(xP, Q) e(yP, Q), x + y = ac (or not)
            x = rng.randrange(1, b.R)
            y = (a * c - x) % b.R if case == 4 else (a * c - x + 5) % b.R
            terms = [terms[0], (b.g1_neg(b.g1_mul(g1, x)), g2), (b.g1_neg(b.g1_mul(g1, y)), g2)]
        f = b.F12_ONE
        for p, q in terms:
            f = b.f12mul(f, b.miller_loop(p, q))
        holds = b.final_exponentiation(f) == b.F12_ONE
        eqs.append({"g1": [b.g1_bytes(p).hex() for p, _ in terms], "g2": [b.g2_bytes(q).hex() for _, q in terms],
                    "holds": holds})
    with open(OUT, "w") as fh:
        json.dump({"single": single, "equations": eqs,
                   "note": "pure-Python optimal ate pairing (tests/golden/bn254_py.py); GT in tower order "
                           "c0.c0.c0 .. c1.c2.c1, canonical 32-byte LE Fq"}, fh, indent=1)
    print(OUT, len(single), "pairings,", len(eqs), "equations:", [e["holds"] for e in eqs])


if __name__ == "__main__":
    main()
