"""Pins the C++ oracle against the golden vectors (CPU only).

The golden vectors come from tests/golden/make_golden.py (pure-Python
affine arithmetic) and restate the reference's known-answer tests:
ntt_backend.rs:63-86, icicle_backend.rs:83-129, sparse_msm_backend.rs,
g2_validation/tests.rs:17-57 and codec.rs:36-101.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import bn254_py as b  # noqa: E402

H = bytes.fromhex


def test_constants_pin_arkworks_orientation(golden):
    c = golden["constants"]
    # ark-bn254 0.4.0 Fr TWO_ADIC_ROOT_OF_UNITY (published constant) equals
    # GENERATOR^((r-1)/2^28) with GENERATOR = 5.
    published = 19103219067921713944291392827692070036145651957329286315305642004821462161904
    assert int.from_bytes(H(c["two_adic_root"]), "little") == published
    w = int.from_bytes(H(c["root_2_20"]), "little")
    assert pow(w, 1 << 19, b.R) == b.R - 1
    assert pow(w, 1 << 20, b.R) == 1


@pytest.mark.parametrize("naive", [True, False])
def test_g1_msm_matches_golden(golden, oracle, naive):
    for case in golden["msm_g1"]:
        pts = b"".join(H(p) for p in case["points"])
        scs = b"".join(H(s) for s in case["scalars"])
        assert oracle.msm_g1(pts, scs, naive=naive).hex() == case["expected"], case["name"]


def test_g1_msm_pippenger_path_on_larger_inputs(golden, oracle):
    # 64 copies of G times 3 exercises the Pippenger branch (n >= 32).
    case = next(c for c in golden["msm_g1"] if c["name"] == "repeated_g_times_3")
    pts = b"".join(H(p) for p in case["points"])
    scs = b"".join(H(s) for s in case["scalars"])
    assert oracle.msm_g1(pts, scs, naive=False).hex() == case["expected"]
    # Pippenger and naive agree on a seeded 300-point case.
    pts, _ = oracle.srs_g1(5, 300)
    scs = oracle.uniform_fr(6, 300)
    assert oracle.msm_g1(pts, scs, naive=False) == oracle.msm_g1(pts, scs, naive=True)


def test_sparse_msm_matches_golden(golden, oracle):
    for case in golden["sparse_g1"]:
        bases = b"".join(H(p) for p in case["bases"])
        idx = [e[0] for e in case["entries"]]
        vals = b"".join(H(e[1]) for e in case["entries"])
        assert oracle.sparse_msm_g1(bases, idx, vals).hex() == case["expected"], case["name"]


def test_ntt_matches_golden(golden, oracle):
    for case in golden["ntt"]:
        vals = b"".join(H(v) for v in case["input"])
        out = oracle.ntt(vals, case["kind"])
        exp = b"".join(H(v) for v in case["expected"])
        assert out == exp, case["name"]


def test_ntt_roundtrip_and_invalid_lengths(oracle):
    vals = oracle.uniform_fr(11, 1024)
    for fwd, inv in (("forward", "inverse"), ("coset_forward", "coset_inverse")):
        assert oracle.ntt(oracle.ntt(vals, fwd), inv) == vals
    for n in (3, 17):
        with pytest.raises(ValueError):
            oracle.ntt(bytes(32 * n), "forward")


def test_g2_msm_matches_golden(golden, oracle):
    for case in golden["msm_g2"]:
        pts = b"".join(H(p) for p in case["points"])
        scs = b"".join(H(s) for s in case["scalars"])
        assert oracle.msm_g2(pts, scs).hex() == case["expected"], case["name"]


def test_fixed_base_matches_golden(golden, oracle):
    for key, fn, size in (("fixed_base_g1", oracle.fixed_base_g1, 64), ("fixed_base_g2", oracle.fixed_base_g2, 128)):
        case = golden[key]
        scs = b"".join(H(s) for s in case["scalars"])
        out = fn(scs)
        got = [out[i:i + size].hex() for i in range(0, len(out), size)]
        assert got == case["expected"], key


@pytest.mark.parametrize("algorithm", [1, 2, 3])
def test_g2_check_matches_golden(golden, oracle, algorithm):
    wire = b"".join(H(w) for w in golden["g2_check"]["wire"])
    masks = oracle.g2_check(wire, algorithm)
    assert masks.tolist() == golden["g2_check"]["masks"]


def test_chacha_stream_matches_python(oracle):
    rng = b.ChaCha20Stream(123)
    expect = b"".join(b.fe_bytes(rng.uniform(b.R)) for _ in range(40))
    assert oracle.uniform_fr(123, 40) == expect
    rng = b.ChaCha20Stream(124)
    expect = b"".join(b.fe_bytes(rng.uniform(b.Q)) for _ in range(40))
    assert oracle.uniform_fq(124, 40) == expect


def test_twist_points_are_on_curve_and_mostly_outside_subgroup(oracle):
    pts = oracle.g2_twist_points(1720001, 8)
    for i in range(8):
        p = pts[128 * i:128 * i + 128]
        assert oracle.g2_on_curve(p)
    masks = oracle.g2_check(pts, 3)
    assert (masks == 4).all()


def test_codec_rejections(golden, oracle):
    for bad in golden["codec"]["g1_reject"]:
        assert not oracle.g1_on_curve(H(bad))
    # non-canonical scalars are rejected by the NTT input decoder
    for bad in golden["codec"]["fr_reject"]:
        with pytest.raises(ValueError):
            oracle.ntt(H(bad), "forward")
    for good in golden["codec"]["fr_accept"]:
        assert oracle.ntt(H(good), "forward") == H(good)


def test_oracle_g1_fft_is_the_dft(oracle):
    """The oracle's G1 transform (arkworks radix-2 FFT over G1, operators.rs:
    413-440) equals the DFT definition out_i = sum_j w^(ij) P_j, one MSM per
    output, with w the pinned arkworks root; inverse scales by 1/n."""
    R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
    root28 = 0x2A3C09F0A58A7E8500E0A7EB8EF62ABC402D111E41112ED49BD61B6E725B19F0
    for n in (1, 2, 4, 8):
        pts, _ = oracle.srs_g1(33 + n, n)
        w = pow(root28, 2 ** (28 - (n.bit_length() - 1)), R)
        for inverse in (False, True):
            got = oracle.g1_fft(pts, n, inverse)
            ww = pow(w, R - 2, R) if inverse else w
            scale = pow(n, R - 2, R) if inverse else 1
            for i in range(n):
                sc = b"".join((pow(ww, i * j, R) * scale % R).to_bytes(32, "little") for j in range(n))
                assert got[64 * i:64 * (i + 1)] == oracle.msm_g1(pts, sc), (n, inverse, i)
