"""NTT, fixed-base and batched G2 validation parity on the GPU.

Mirrors crates/gpu/tests/ntt_backend.rs (known values, sizes 1..16384,
forward/inverse, round trips, invalid lengths), setup_tables.rs /
fixed_base_cpu.rs, and g2_validation/tests.rs (wire corpus, masks 1/2/4,
all three subgroup algorithms).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = bytes.fromhex


def test_golden_ntt(backend, golden):
    for case in golden["ntt"]:
        vals = b"".join(H(v) for v in case["input"])
        exp = b"".join(H(v) for v in case["expected"])
        kind = case["kind"]
        if kind.startswith("coset"):
            got = backend.ntt_coset(vals, inverse=kind.endswith("inverse"))
        else:
            got = backend.ntt(vals, inverse=kind == "inverse")
        assert got == exp, case["name"]


@pytest.mark.parametrize("kind", ["forward", "inverse", "coset_forward", "coset_inverse"])
def test_ntt_matches_oracle_across_sizes(backend, oracle, kind):
    for logn in range(0, 15):
        n = 1 << logn
        vals = bytearray(oracle.uniform_fr(7000 + logn, n))
        vals[0:32] = (0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000000).to_bytes(32, "little")
        vals = bytes(vals)
        if kind.startswith("coset"):
            got = backend.ntt_coset(vals, inverse=kind.endswith("inverse"))
        else:
            got = backend.ntt(vals, inverse=kind == "inverse")
        assert got == oracle.ntt(vals, kind), f"n={n} {kind}"


def test_ntt_reference_root_abi(backend, golden, oracle):
    root = H(golden["constants"]["root_2_20"])
    vals = oracle.uniform_fr(42, 1024)
    assert backend.ntt_with_root(vals, False, root) == oracle.ntt(vals, "forward")
    bad_root = (5).to_bytes(32, "little")
    with pytest.raises(Exception):
        backend.ntt_with_root(vals, False, bad_root)
    # a root of order 2^20 defines no longer transform: the reference's cap
    with pytest.raises(Exception):
        backend.ntt_with_root(bytes(32 << 21), False, root)
    assert backend.ntt_with_root(vals, False, root) == oracle.ntt(vals, "forward")  # owner still healthy


def test_ntt_roundtrip_large_and_invalid_lengths(backend, oracle, dv):
    for logn in (16, 20, 22):
        n = 1 << logn
        vals = oracle.uniform_fr(8000 + logn, n)
        for fwd, inv in ((False, True),):
            assert backend.ntt(backend.ntt(vals, fwd), inv) == vals
        assert backend.ntt_coset(backend.ntt_coset(vals, False), True) == vals
    for n in (3, 17):
        with pytest.raises(ValueError):
            backend.ntt(bytes(32 * n), False)
    with pytest.raises(dv.DvgpuError):
        backend.ntt(bytes([0xFF]) * 32 * 4, False)
    ones = (1).to_bytes(32, "little") * 16
    got = backend.ntt(ones, False)
    assert got[:32] == (16).to_bytes(32, "little") and got[32:] == bytes(32 * 15)


def test_ntt_2_16_matches_oracle(backend, oracle):
    vals = oracle.uniform_fr(1616, 1 << 16)
    for kind in ("forward", "inverse", "coset_forward"):
        if kind.startswith("coset"):
            got = backend.ntt_coset(vals, inverse=False)
        else:
            got = backend.ntt(vals, inverse=kind == "inverse")
        assert got == oracle.ntt(vals, kind), kind


def test_golden_fixed_base(backend, golden):
    for key, fn, size in (("fixed_base_g1", backend.fixed_base_g1, 64), ("fixed_base_g2", backend.fixed_base_g2, 128)):
        case = golden[key]
        scs = b"".join(H(s) for s in case["scalars"])
        out = fn(scs)
        assert [out[i:i + size].hex() for i in range(0, len(out), size)] == case["expected"], key


def test_fixed_base_matches_oracle(backend, oracle):
    for n in (1, 31, 32, 33, 1000, 5000):
        sc = oracle.uniform_fr(10 + n, n)
        assert backend.fixed_base_g1(sc) == oracle.fixed_base_g1(sc), n
    for n in (1, 33, 700):
        sc = oracle.uniform_fr(20 + n, n)
        assert backend.fixed_base_g2(sc) == oracle.fixed_base_g2(sc), n


def test_fixed_base_chunked_calls(backend, oracle, dv):
    """Calls longer than one 2^17-point chunk (generation of a chunk overlaps
    the host copy of the previous one), and a non-canonical scalar in a
    later chunk: the call fails and writes no output."""
    n = (1 << 17) + 1000
    sc = oracle.uniform_fr(31, n)
    assert backend.fixed_base_g1(sc) == oracle.fixed_base_g1(sc)
    sc2 = sc[:32 * 70000]
    assert backend.fixed_base_g2(sc2 + sc[32 * 131000:32 * 131100]) == \
        oracle.fixed_base_g2(sc2 + sc[32 * 131000:32 * 131100])
    bad = bytearray(sc)
    bad[32 * 131500:32 * 131501] = b"\xff" * 32           # >= r, in the second chunk
    out = ctypes.create_string_buffer(b"\xab" * (n * 64), n * 64)
    err = ctypes.create_string_buffer(256)
    rc = dv.lib().dvgpu_bn254_fixed_base(backend.handle, bytes(bad), n, 0, out, err, 256)
    assert rc == -1 and b"131500" in err.value
    assert out.raw == b"\xab" * (n * 64)


@pytest.mark.parametrize("algorithm", [1, 2, 3])
def test_golden_g2_validation(backend, golden, algorithm):
    wire = b"".join(H(w) for w in golden["g2_check"]["wire"])
    masks, rep = backend.inspect_g2_validation(wire, algorithm)
    exp = golden["g2_check"]["masks"]
    assert masks.tolist() == exp
    bad = [i for i, m in enumerate(exp) if m]
    assert rep.checked_points == len(exp) and rep.invalid_points == len(bad)
    assert rep.first_invalid == bad[0] and rep.algorithm == algorithm
    mask = 0
    for m in exp:
        mask |= m
    assert rep.failure_mask == mask


@pytest.mark.parametrize("algorithm", [1, 2, 3])
def test_g2_validation_mixed_corpus_matches_oracle(backend, oracle, algorithm):
    valid = oracle.fixed_base_g2(oracle.uniform_fr(1720002, 256))
    twist = oracle.g2_twist_points(1720001, 256)
    wire = valid + twist
    masks, rep = backend.inspect_g2_validation(wire, algorithm)
    assert masks.tolist() == oracle.g2_check(wire, algorithm).tolist()
    assert (masks[:256] == 0).all() and (masks[256:] == 4).all()
    assert rep.first_invalid == 256 and rep.invalid_points == 256 and rep.failure_mask == 4
    empty_masks, empty = backend.inspect_g2_validation(b"", algorithm)
    assert empty.checked_points == 0 and empty.first_invalid == 2**64 - 1


def test_fixed_base_g2_checked(backend, oracle, dv):
    sc = oracle.uniform_fr(99, 300)
    out, rep = backend.fixed_base_g2_checked(sc, 3)
    assert out == oracle.fixed_base_g2(sc)
    assert rep.invalid_points == 0 and rep.first_invalid == 2**64 - 1 and rep.checked_points == 300


def test_random_twist_points_are_off_subgroup(backend, oracle):
    """The device corpus generator: every point parses, lies on the twist
    curve and (no cofactor clearing) fails the subgroup check -- mask 4 in
    the oracle and on the GPU, for every algorithm."""
    import torch
    n = 300
    d = torch.empty(n * 128, dtype=torch.uint8, device="cuda")
    backend.random_twist_device(99, n, d.data_ptr())
    torch.cuda.synchronize()
    wire = d.cpu().numpy().tobytes()
    assert len(set(wire[128 * i:128 * (i + 1)] for i in range(n))) == n
    for alg in (1, 2, 3):
        expect = oracle.g2_check(wire, alg)
        assert (expect == 4).all(), alg
        masks, rep = backend.inspect_g2_validation(wire, alg)
        assert (masks == expect).all() and rep.invalid_points == n, alg
