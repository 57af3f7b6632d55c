"""Generate tests/golden/golden.json from the pure-Python BN254 restatement.

Run from the repository root:  python tests/golden/make_golden.py

The vectors are the reference's own known-answer tests, restated, plus
small seeded cases that are computed here with plain affine Python-integer
arithmetic:

* NTT impulse / constant / roundtrip: crates/gpu/tests/ntt_backend.rs:63-86.
* MSM [3]G, G + (-G), zero scalars, N copies of G times 3:
  crates/gpu/tests/icicle_backend.rs:83-91,114-129.
* Sparse 17 x (5 G) = [85]G and repeated/zero entries:
  crates/gpu/tests/sparse_msm_backend.rs:18-45,69-87.
* G2 wire corpus (flags, modulus +-1, +-generator, twist points):
  crates/gpu/src/g2_validation/tests.rs:17-57.
* Codec rejection: crates/gpu/tests/codec.rs:36-101.

Random cases use identity points every 7th index and zero scalars every 11th,
as icicle_backend.rs:72-80 does.  Seeds are ChaCha20 stream seeds (key = seed
as u64 LE); they are this project's seeds, not rand_chacha's StdRng streams.
"""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import bn254_py as b  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def hx(data):
    return data.hex()


def fr_hex(v):
    return hx(b.fe_bytes(v))


def g1_case(name, points, scalars):
    acc = None
    for p, s in zip(points, scalars):
        acc = b.g1_add(acc, b.g1_mul(p, s))
    return {"name": name, "points": [hx(b.g1_bytes(p)) for p in points],
            "scalars": [fr_hex(s) for s in scalars], "expected": hx(b.g1_bytes(acc))}


def g2_case(name, points, scalars):
    acc = None
    for p, s in zip(points, scalars):
        acc = b.g2_add(acc, b.g2_mul(p, s))
    return {"name": name, "points": [hx(b.g2_bytes(p)) for p in points],
            "scalars": [fr_hex(s) for s in scalars], "expected": hx(b.g2_bytes(acc))}


def main():
    out = {"generator": "tests/golden/make_golden.py"}
    G, G2 = b.G1_GEN, b.G2_GEN
    assert b.g1_on_curve(G) and b.g2_on_curve(G2)
    assert b.g1_mul(G, b.R) is None and b.g2_mul(G2, b.R) is None

    # ------------------------------------------------------------ constants
    out["constants"] = {
        "q": hex(b.Q), "r": hex(b.R),
        "two_adic_root": fr_hex(b.root_of_unity(1 << 28)),
        "root_2_20": fr_hex(b.root_of_unity(1 << 20)),
        "g2_b": [hex(b.B2[0]), hex(b.B2[1])],
        "psi_cx": [hex(b.PSI_CX[0]), hex(b.PSI_CX[1])],
        "psi_cy": [hex(b.PSI_CY[0]), hex(b.PSI_CY[1])],
    }

    # ------------------------------------------------------------ G1 MSM
    msm = []
    msm.append(g1_case("three_g", [G], [3]))
    msm.append(g1_case("g_plus_neg_g", [G, G], [1, b.R - 1]))
    msm.append(g1_case("repeated_g_times_3", [G] * 64, [3] * 64))
    for seed in (7, 17, 2026):
        rng = b.ChaCha20Stream(seed)
        for n in (1, 2, 17, 64):
            pts, scs = [], []
            for i in range(n):
                k = rng.uniform(b.R)
                pts.append(None if i % 7 == 0 else b.g1_mul(G, k))
                scs.append(0 if i % 11 == 0 else rng.uniform(b.R))
            msm.append(g1_case(f"seed{seed}_n{n}", pts, scs))
            msm.append(g1_case(f"seed{seed}_n{n}_zero_scalars", pts, [0] * n))
    # full-width extremes: r-1, 2^253 .. and opposite points
    rng = b.ChaCha20Stream(99)
    pts = [b.g1_mul(G, rng.uniform(b.R)) for _ in range(6)]
    pts += [b.g1_neg(p) for p in pts[:3]]
    scs = [b.R - 1, (1 << 253), (1 << 253) - 1, 1, 2, b.R - 2, 5, 5, 5]
    msm.append(g1_case("extremes_and_opposites", pts, scs))
    out["msm_g1"] = msm

    # ------------------------------------------------------------ sparse MSM
    sparse = []
    sparse.append({"name": "seventeen_times_five_g", "bases": [hx(b.g1_bytes(G))],
                   "entries": [[0, fr_hex(5)]] * 17, "expected": hx(b.g1_bytes(b.g1_mul(G, 85)))})
    rng = b.ChaCha20Stream(2026102201)
    bases = [b.g1_mul(G, rng.uniform(b.R)) for _ in range(97)]
    entries = [((37 * i + 11) % 97, rng.uniform(b.R)) for i in range(53)]
    for name, bs, es in (
        ("indexed53", bases, entries),
        ("indexed53_opposite", [b.g1_neg(p) for p in bases], entries),
        ("repeated_zero", bases, [(96, 9), (0, 0), (96, b.R - 2)]),
        ("empty", bases, []),
    ):
        acc = None
        for idx, v in es:
            acc = b.g1_add(acc, b.g1_mul(bs[idx], v))
        sparse.append({"name": name, "bases": [hx(b.g1_bytes(p)) for p in bs],
                       "entries": [[i, fr_hex(v)] for i, v in es], "expected": hx(b.g1_bytes(acc))})
    out["sparse_g1"] = sparse

    # ------------------------------------------------------------ NTT
    ntt = []
    ntt.append({"name": "impulse8", "kind": "forward", "input": [fr_hex(1)] + [fr_hex(0)] * 7,
                "expected": [fr_hex(1)] * 8})
    ntt.append({"name": "const5_8", "kind": "forward", "input": [fr_hex(5)] * 8,
                "expected": [fr_hex(40)] + [fr_hex(0)] * 7})
    ntt.append({"name": "const5_8_inverse", "kind": "inverse", "input": [fr_hex(40)] + [fr_hex(0)] * 7,
                "expected": [fr_hex(5)] * 8})
    ntt.append({"name": "ones16", "kind": "forward", "input": [fr_hex(1)] * 16,
                "expected": [fr_hex(16)] + [fr_hex(0)] * 15})
    for seed in (7, 17, 2026):
        rng = b.ChaCha20Stream(seed + 1000)
        for n in (1, 2, 4, 8, 16, 64, 256):
            vals = [rng.uniform(b.R) for _ in range(n)]
            vals[0] = b.R - 1
            for kind in ("forward", "inverse", "coset_forward", "coset_inverse"):
                exp = b.dft(vals, inverse=kind.endswith("inverse"), coset=kind.startswith("coset"))
                ntt.append({"name": f"seed{seed}_n{n}_{kind}", "kind": kind,
                            "input": [fr_hex(v) for v in vals], "expected": [fr_hex(v) for v in exp]})
    out["ntt"] = ntt

    # ------------------------------------------------------------ G2 MSM
    msm2 = [g2_case("three_g2", [G2], [3]), g2_case("g2_plus_neg", [G2, G2], [1, b.R - 1])]
    rng = b.ChaCha20Stream(4242)
    for n in (1, 3, 8):
        pts = [None if i % 7 == 0 else b.g2_mul(G2, rng.uniform(b.R)) for i in range(n)]
        scs = [0 if i % 11 == 0 else rng.uniform(b.R) for i in range(n)]
        msm2.append(g2_case(f"random_n{n}", pts, scs))
    out["msm_g2"] = msm2

    # ------------------------------------------------------------ fixed base
    rng = b.ChaCha20Stream(31337)
    fscal = [0, 1, 2, 3, 15, 16, 255, 256, b.R - 1, (1 << 253) + 12345] + [rng.uniform(b.R) for _ in range(6)]
    out["fixed_base_g1"] = {"scalars": [fr_hex(s) for s in fscal],
                            "expected": [hx(b.g1_bytes(b.g1_mul(G, s))) for s in fscal]}
    out["fixed_base_g2"] = {"scalars": [fr_hex(s) for s in fscal],
                            "expected": [hx(b.g2_bytes(b.g2_mul(G2, s))) for s in fscal]}

    # ------------------------------------------------------------ G2 check corpus
    corpus = [bytes(128)]
    for p in (G2, b.g2_neg(G2)):
        w = b.g2_bytes(p)
        corpus.append(w)
        for flag in (0, 0x40, 0x80, 0xC0):
            c = bytearray(w); c[127] |= flag; corpus.append(bytes(c))
        for i in range(0, 128, 3):
            c = bytearray(w); c[i] ^= 0x80; corpus.append(bytes(c))
    for flag in (0x40, 0x80, 0xC0):
        c = bytearray(128); c[127] = flag; corpus.append(bytes(c))
    for field in range(4):
        for adj in (-1, 0, 1):
            c = bytearray(b.g2_bytes(G2))
            c[32 * field:32 * field + 32] = (b.Q + adj).to_bytes(32, "little")
            corpus.append(bytes(c))
    rng = b.ChaCha20Stream(1720001)
    twist = []
    while len(twist) < 24:
        p = b.twist_point_from_x((rng.uniform(b.Q), rng.uniform(b.Q)))
        if p is not None:
            twist.append(p)
    for p in twist:
        corpus.append(b.g2_bytes(p))
    for p in twist[:4]:
        qq = b.g2_mul(p, b.R)  # pure cofactor component: on curve, outside G2
        corpus.append(b.g2_bytes(qq))
        corpus.append(b.g2_bytes(b.g2_add(qq, G2)))
    for _ in range(8):
        corpus.append(b.g2_bytes(b.g2_mul(G2, rng.uniform(b.R))))
    masks = [b.g2_wire_mask(c) for c in corpus]
    # the three predicates must agree on every on-curve point
    for c, m in zip(corpus, masks):
        for pred in (b.subgroup_frobenius_127, b.subgroup_frobenius_63):
            assert b.g2_wire_mask(c, pred) == m
    assert 0 in masks and 1 in masks and 2 in masks and 4 in masks
    out["g2_check"] = {"wire": [hx(c) for c in corpus], "masks": masks}

    # ------------------------------------------------------------ codec
    out["codec"] = {
        "fr_reject": [hx(bytes([0xFF] * 32)), fr_hex(b.R)],
        "fr_accept": [fr_hex(b.R - 1), fr_hex(0), fr_hex(2**64 - 1)],
        "g1_reject": [hx(bytes([1] + [0] * 31 + [1] + [0] * 31))],
    }

    with open(OUT, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
