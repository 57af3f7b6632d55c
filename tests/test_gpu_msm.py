"""G1/G2 MSM, batch and sparse MSM parity on the GPU through the C-ABI.

Mirrors crates/gpu/tests/icicle_backend.rs:65-129 (sizes, identity points
every 7th index, zero scalars every 11th, [3]G, G + (-G), repeated bases)
and crates/gpu/tests/sparse_msm_backend.rs / batch_backend.rs.  The
expected values come from the CPU oracle and the golden vectors; results
must be byte-identical.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = bytes.fromhex


def _case_inputs(oracle, seed, n, g2=False):
    size = 128 if g2 else 64
    pts = bytearray((oracle.fixed_base_g2 if g2 else oracle.fixed_base_g1)(oracle.uniform_fr(seed, n)))
    scs = bytearray(oracle.uniform_fr(seed + 1, n))
    for i in range(0, n, 7):
        pts[i * size:(i + 1) * size] = bytes(size)
    for i in range(0, n, 11):
        scs[i * 32:(i + 1) * 32] = bytes(32)
    return bytes(pts), bytes(scs)


def test_golden_g1_msm(backend, golden):
    for case in golden["msm_g1"]:
        pts = b"".join(H(p) for p in case["points"])
        scs = b"".join(H(s) for s in case["scalars"])
        assert backend.msm(pts, scs).hex() == case["expected"], case["name"]


@pytest.mark.parametrize("seed", [7, 17, 2026])
def test_g1_msm_matches_oracle_across_sizes(backend, oracle, seed):
    for n in [0, 1, 2, 17, 511, 512, 1023, 1024, 2048, 6144, 8192]:
        pts, scs = _case_inputs(oracle, seed * 100 + n, n)
        expect = oracle.msm_g1(pts, scs)
        assert backend.msm(pts, scs) == expect, f"seed={seed} n={n}"
        assert backend.msm(pts, bytes(32 * n)) == bytes(64)
        assert backend.msm(pts, scs) == expect  # repeat: workspace reuse


def test_g1_msm_every_window_width(backend, oracle):
    pts, scs = _case_inputs(oracle, 555, 3000)
    expect = oracle.msm_g1(pts, scs)
    for c in range(4, 17):
        backend.set_window(c)
        try:
            assert backend.msm(pts, scs) == expect, f"c={c}"
        finally:
            backend.set_window(0)


def test_g1_msm_one_bucket_skew(backend, oracle):
    # every scalar equal: all entries of a window land in one bucket
    g = oracle.fixed_base_g1((1).to_bytes(32, "little"))
    for n in (1024, 8192):
        pts = g * n
        scs = (3).to_bytes(32, "little") * n
        expect = oracle.fixed_base_g1((3 * n).to_bytes(32, "little"))
        assert backend.msm(pts, scs) == expect


def test_g1_msm_2_16_matches_oracle(backend, oracle):
    n = 1 << 16
    pts, tau = oracle.srs_g1(2812, n)
    scs = oracle.uniform_fr(2813, n)
    assert backend.msm(pts, scs) == oracle.msm_g1(pts, scs)


def test_g1_msm_rejects_invalid_inputs_and_stays_healthy(backend, dv, oracle):
    pts, scs = _case_inputs(oracle, 9, 64)
    bad_point = bytearray(pts)
    bad_point[64 * 5:64 * 6] = (1).to_bytes(32, "little") + (1).to_bytes(32, "little")  # (1,1) off curve
    with pytest.raises(dv.DvgpuError) as e:
        backend.msm(bytes(bad_point), scs)
    assert e.value.status == -1
    bad_scalar = bytearray(scs)
    bad_scalar[32 * 3:32 * 4] = bytes([0xFF] * 32)
    with pytest.raises(dv.DvgpuError) as e:
        backend.msm(pts, bytes(bad_scalar))
    assert e.value.status == -1
    assert backend.msm(pts, scs) == oracle.msm_g1(pts, scs)


def test_golden_g2_msm(backend, golden):
    for case in golden["msm_g2"]:
        pts = b"".join(H(p) for p in case["points"])
        scs = b"".join(H(s) for s in case["scalars"])
        assert backend.msm_g2_host(pts, scs).hex() == case["expected"], case["name"]


def test_g2_msm_matches_oracle(backend, oracle):
    for n in [0, 1, 2, 17, 300, 1024, 4096]:
        pts, scs = _case_inputs(oracle, 4000 + n, n, g2=True)
        assert backend.msm_g2_host(pts, scs) == oracle.msm_g2(pts, scs), f"n={n}"


def test_padded_batch_matches_per_set_results(backend, oracle):
    length, count = 200, 5
    pts, scs = _case_inputs(oracle, 31, length * count)
    got = backend.msm_batch_padded(pts, scs, length, count)
    for k in range(count):
        sl = slice(k * length, (k + 1) * length)
        assert got[k] == oracle.msm_g1(pts[sl.start * 64:sl.stop * 64], scs[sl.start * 32:sl.stop * 32])


def test_uneven_batch_and_shared_scalars(backend, oracle):
    sizes = [0, 1, 5, 300, 17, 2048, 3]
    pts, scs = _case_inputs(oracle, 77, sum(sizes))
    offs = np.concatenate([[0], np.cumsum(sizes)]).tolist()
    got = backend.msm_batch_uneven(pts, scs, offs)
    for k in range(len(sizes)):
        a, b = offs[k], offs[k + 1]
        assert got[k] == oracle.msm_g1(pts[a * 64:b * 64], scs[a * 32:b * 32]), f"set {k}"
    # BatchMsmRequest form: point sets sharing one scalar vector
    sets = [pts[:64 * 10], pts[64 * 10:64 * 40]]
    got = backend.msm_batch(sets, scs, offsets=[0, 5], lengths=[10, 30])
    assert got[0] == oracle.msm_g1(pts[:640], scs[:320])
    assert got[1] == oracle.msm_g1(pts[640:64 * 40], scs[160:160 + 960])


def test_uneven_batch_with_long_reduction_segments(backend, oracle):
    """128 sets of 2^15 points: the batch's window model picks c = 11, so the
    launch holds 128 x 24 x 2^10 = 3.1 M buckets and the bucket reduction
    takes 16-bucket segments (2^21 buckets or more) instead of 8.  Every set
    is compared with the oracle."""
    from concurrent.futures import ThreadPoolExecutor
    count, n = 128, 1 << 15
    base, _ = oracle.srs_g1(7700, n)
    scs = oracle.uniform_fr(7701, count * n)
    offs = [k * n for k in range(count + 1)]
    got = backend.msm_batch_uneven(base * count, scs, offs)
    with ThreadPoolExecutor(8) as pool:
        want = list(pool.map(lambda k: oracle.msm_g1(base, scs[32 * k * n:32 * (k + 1) * n]), range(count)))
    for k in range(count):
        assert got[k] == want[k], f"set {k}"


def test_golden_sparse(backend, golden):
    reqs, expect = [], []
    for case in golden["sparse_g1"]:
        bases = b"".join(H(p) for p in case["bases"])
        entries = [(e[0], H(e[1])) for e in case["entries"]]
        reqs.append((bases, entries))
        expect.append(case["expected"])
    got = backend.msm_sparse_batch(reqs)
    assert [g.hex() for g in got] == expect
    # 70 copies of 17 x (5 G): splits nothing here, one launch sequence
    seventeen = reqs[0]
    got = backend.msm_sparse_batch([seventeen] * 70)
    assert all(g.hex() == expect[0] for g in got)


def test_sparse_resident_matches_oracle(backend, oracle):
    n = 1 << 14
    bases, _ = oracle.srs_g1(65536, n)
    h = backend.register_bases(bases)
    try:
        rng = np.random.default_rng(5)
        reqs = []
        for k in (16, 256, 1, 0, 1000):
            idx = rng.choice(n, size=k, replace=False).astype(np.uint64)
            vals = oracle.uniform_fr(900 + k, k)
            reqs.append((idx, vals))
        # repeated index and zero scalar
        reqs.append((np.array([7, 7, 3], dtype=np.uint64), (9).to_bytes(32, "little") + bytes(32) + (2).to_bytes(32, "little")))
        idx_all = np.concatenate([r[0] for r in reqs]) if reqs else np.zeros(0, np.uint64)
        vals_all = b"".join(r[1] for r in reqs)
        offs = np.concatenate([[0], np.cumsum([len(r[0]) for r in reqs])])
        expect = [oracle.sparse_msm_g1(bases, idx, vals) for idx, vals in reqs]
        got = backend.sparse_msm_resident(h, idx_all, vals_all, offs)
        assert got == expect
        with pytest.raises(Exception):
            backend.sparse_msm_resident(h, np.array([n], dtype=np.uint64), bytes(32), [0, 1])
        # with a table of precomputed window multiples the same requests take
        # the one-bucket-set path (host and device forms)
        import torch
        d_idx = torch.from_numpy(idx_all.view(np.int64)).cuda()
        d_vals = torch.frombuffer(bytearray(vals_all), dtype=torch.uint8).cuda()
        torch.cuda.synchronize()
        for c in (8, 11, 0):
            backend.precompute_bases(h, c)
            assert backend.sparse_msm_resident(h, idx_all, vals_all, offs) == expect, c
            assert backend.sparse_msm_device(h, d_idx.data_ptr(), d_vals.data_ptr(), offs) == expect, c
        bad = torch.tensor([n], dtype=torch.int64, device="cuda")
        with pytest.raises(Exception):
            backend.sparse_msm_device(h, bad.data_ptr(), d_vals.data_ptr(), [0, 1])
        assert backend.sparse_msm_resident(h, idx_all, vals_all, offs) == expect  # owner still healthy
    finally:
        backend.release_bases(h)


def test_sparse_direct_small_supports(backend, oracle, dv):
    """Small sparse requests over a table of window multiples take the direct
    path (one thread per entry and window, no bucket sort): results equal the
    oracle's for repeated indices, zero scalars, empty requests and many tiny
    requests, on both sides of the size limit, and bad inputs are rejected
    with the owner left healthy."""
    import torch
    n = 1 << 12
    bases, _ = oracle.srs_g1(4096, n)
    h = backend.register_bases(bases)
    try:
        rng = np.random.default_rng(11)
        sizes = [16, 1, 0, 3, 40] + [2] * 20
        reqs = []
        for j, k in enumerate(sizes):
            idx = rng.choice(n, size=k, replace=False).astype(np.uint64)
            reqs.append((idx, oracle.uniform_fr(1200 + j, k)))
        reqs.append((np.array([5, 5, 9], dtype=np.uint64), (3).to_bytes(32, "little") + bytes(32) + (7).to_bytes(32, "little")))
        idx_all = np.concatenate([r[0] for r in reqs])
        vals_all = b"".join(r[1] for r in reqs)
        offs = np.concatenate([[0], np.cumsum([len(r[0]) for r in reqs])])
        expect = [oracle.sparse_msm_g1(bases, idx, vals) for idx, vals in reqs]
        for c in (8, 11, 0):
            backend.precompute_bases(h, c)
            assert backend.sparse_msm_resident(h, idx_all, vals_all, offs) == expect, c
            d_idx = torch.from_numpy(idx_all.view(np.int64)).cuda()
            d_vals = torch.frombuffer(bytearray(vals_all), dtype=torch.uint8).cuda()
            assert backend.sparse_msm_device(h, d_idx.data_ptr(), d_vals.data_ptr(), offs) == expect, c
        # just below and above the direct path's limit (c = 8: 32 windows, 2^16 terms)
        backend.precompute_bases(h, 8)
        for k in (512, 2048, 2049):
            idx = rng.choice(n, size=k, replace=False).astype(np.uint64)
            vals = oracle.uniform_fr(1300 + k, k)
            assert backend.sparse_msm_resident(h, idx, vals, [0, k]) == [oracle.sparse_msm_g1(bases, idx, vals)]
        bad_idx = torch.tensor([1, n], dtype=torch.int64, device="cuda")
        two = torch.frombuffer(bytearray(oracle.uniform_fr(1400, 2)), dtype=torch.uint8).cuda()
        with pytest.raises(dv.DvgpuError) as e:
            backend.sparse_msm_device(h, bad_idx.data_ptr(), two.data_ptr(), [0, 2])
        assert e.value.status == -1 and "out of range" in e.value.message
        r_mod = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
        with pytest.raises(dv.DvgpuError) as e:
            backend.sparse_msm_resident(h, np.array([1, 2], dtype=np.uint64), bytes(32) + r_mod.to_bytes(32, "little"),
                                        [0, 2])
        assert e.value.status == -1 and "non-canonical scalar at index 1" in e.value.message
        assert backend.sparse_msm_resident(h, idx_all, vals_all, offs) == expect  # owner still healthy
    finally:
        backend.release_bases(h)


def test_autotune_picks_a_window_and_results_stay_exact(dv, oracle):
    with dv.DvgpuBackend() as b:
        c, log = b.autotune_msm(4096)
        assert 4 <= c <= 20 and log["best_c"] == c and len(log["candidates"]) >= 3
        assert b.window_for(4096) == c
        pts, scs = _case_inputs(oracle, 4242, 4000)
        assert b.msm(pts, scs) == oracle.msm_g1(pts, scs)
        c2, _ = b.autotune_msm(1000, g2=True)
        pts2, scs2 = _case_inputs(oracle, 4343, 1000, g2=True)
        assert b.msm_g2_host(pts2, scs2) == oracle.msm_g2(pts2, scs2)


def test_skewed_digits_long_bucket_chains(backend, oracle):
    """Buckets that span thousands of accumulation slices (every scalar equal)
    and tiny top windows (c = 14 and 18 leave 2 bits in the top window)."""
    n = 1 << 17
    pts, _ = oracle.srs_g1(1717, n)
    same = oracle.uniform_fr(1718, 1) * n
    assert backend.msm(pts, same) == oracle.msm_g1(pts, same)
    top = b"".join((((1 << 253) + (i % 3)) % (1 << 254)).to_bytes(32, "little") for i in range(n))
    expect = oracle.msm_g1(pts, top)
    rnd = oracle.uniform_fr(1719, n)
    expect_rnd = oracle.msm_g1(pts, rnd)
    for c in (14, 18):
        backend.set_window(c)
        try:
            assert backend.msm(pts, top) == expect, f"c={c}"
            assert backend.msm(pts, rnd) == expect_rnd, f"c={c}"
        finally:
            backend.set_window(0)


def test_precomputed_resident_msm_matches_oracle(backend, oracle):
    import torch
    n = 1 << 14
    pts, _ = oracle.srs_g1(777, n)
    scs = oracle.uniform_fr(778, n)
    expect = oracle.msm_g1(pts, scs)
    expect_prefix = oracle.msm_g1(pts[:1000 * 64], scs[:1000 * 32])
    d_sc = torch.frombuffer(bytearray(scs), dtype=torch.uint8).cuda()
    torch.cuda.synchronize()
    h = backend.register_bases(pts)
    try:
        assert backend.msm_resident(h, d_sc.data_ptr(), n) == expect
        for c in (0, 8, 13, 16):
            backend.precompute_bases(h, c)
            assert backend.msm_resident(h, d_sc.data_ptr(), n) == expect, f"c={c}"
            assert backend.msm_resident(h, d_sc.data_ptr(), 1000) == expect_prefix, f"c={c} prefix"
    finally:
        backend.release_bases(h)
    pts2, scs2 = _case_inputs(oracle, 779, 2000, g2=True)
    d_sc2 = torch.frombuffer(bytearray(scs2), dtype=torch.uint8).cuda()
    torch.cuda.synchronize()
    h2 = backend.register_bases(pts2, g2=True)
    try:
        backend.precompute_bases(h2, 0)
        assert backend.msm_resident(h2, d_sc2.data_ptr(), 2000, g2=True) == oracle.msm_g2(pts2, scs2)
    finally:
        backend.release_bases(h2)


def test_resident_host_msm(backend, oracle, dv):
    """Host-scalar MSMs over registered bases with a precomputed table
    (dvgpu_bn254_msm_resident_host, the e2e call of the headline bench): the
    same result as the oracle and the plain call; a bad scalar late in the
    call is reported with its index and leaves the result untouched."""
    n = (1 << 18) + 3
    pts, _ = oracle.srs_g1(6400, n, threads=16)
    sc = oracle.uniform_fr(6401, n)
    h = backend.register_bases(pts)
    try:
        backend.precompute_bases(h, 0)
        expect = oracle.msm_g1(pts, sc, threads=16)
        assert backend.msm_resident_host(h, sc) == expect == backend.msm(pts, sc)
        m = (1 << 18) - 5
        assert backend.msm_resident_host(h, sc[:32 * m]) == oracle.msm_g1(pts[:64 * m], sc[:32 * m], threads=16)
        bad = bytearray(sc)
        bad[32 * (n - 7):32 * (n - 6)] = b"\xff" * 32
        out = ctypes.create_string_buffer(b"\x5a" * 64, 64)
        err = ctypes.create_string_buffer(256)
        rc = dv.lib().dvgpu_bn254_msm_resident_host(backend.handle, h, bytes(bad), n, out, err, 256)
        assert rc == -1 and str(n - 7).encode() in err.value and out.raw == b"\x5a" * 64
        assert backend.msm_resident_host(h, sc) == expect  # owner still healthy
    finally:
        backend.release_bases(h)
